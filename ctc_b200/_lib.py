"""ctypes binding of libctc_b200.so (the C ABI of include/ctc_b200.h).

The library is the product: if it is missing or fails to load this module
raises -- there is no CPU fallback.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libctc_b200.so")

CTC_OK, CTC_ERR_ARG, CTC_ERR_CUDA, CTC_ERR_CAPACITY, CTC_ERR_DEVICE = 0, 1, 2, 3, 4
CTC_RNG_REFERENCE, CTC_RNG_STABLE = 0, 1
CTC_SIM_PHASES = 9
CTC_BOP_FLOAT, CTC_BOP_INT = 0, 1
CTC_RESTART_TEMPL, CTC_RESTART_FINAL = -1, -2
CTC_WVEL_CSTE, CTC_WVEL_SHEAR, CTC_WVEL_SHEAR_SIN, CTC_WVEL_HS = 0, 1, 2, 3
SIM_PHASE_NAMES = ("clist", "frag_starts", "bulk", "halo", "wall", "fsi", "contact", "update", "membrane")

vp = C.c_void_p
ip = C.POINTER(C.c_int)
fp = C.POINTER(C.c_float)


class DpdParams(C.Structure):
    _fields_ = [("a", C.c_float), ("g", C.c_float), ("s", C.c_float), ("spow", C.c_float)]


class DpdLjParams(C.Structure):
    _fields_ = [("a", C.c_float), ("g", C.c_float), ("s", C.c_float), ("spow", C.c_float),
                ("ljs", C.c_float), ("lje", C.c_float)]


class Wvel(C.Structure):
    """ctc_wvel: the wall velocity (CTC_WVEL_CSTE / SHEAR / SHEAR_SIN / HS)."""
    _fields_ = [("type", C.c_int), ("u", C.c_float * 3), ("gdot", C.c_float), ("vdir", C.c_int), ("gdir", C.c_int),
                ("half", C.c_int), ("w", C.c_float), ("h", C.c_float)]


class RbcParams(C.Structure):
    _fields_ = [(k, C.c_float) for k in
                ("gammaC", "gammaT", "kBT", "kb", "phi", "ks", "x0", "mpow", "ka", "kd", "kv",
                 "totArea", "totVolume")]


class SimConfig(C.Structure):
    _fields_ = [("LX", C.c_int), ("LY", C.c_int), ("LZ", C.c_int), ("maxp", C.c_int),
                ("dpd", DpdParams), ("mass", C.c_float), ("dt", C.c_float),
                ("bodyf", C.c_float * 3), ("rng", C.c_int)]


class SubConfig(C.Structure):
    _fields_ = [("sim", SimConfig), ("dims", C.c_int * 3), ("coords", C.c_int * 3), ("rank", C.c_int),
                ("nbr", C.c_int * 26), ("maxd", C.c_float)]


class BatchConfig(C.Structure):
    _fields_ = [("nbox", C.c_int), ("L", C.POINTER(C.c_int)), ("n", C.POINTER(C.c_int)), ("dpd", DpdParams),
                ("mass", C.c_float), ("dt", C.c_float), ("bodyf", C.c_float * 3), ("rng", C.c_int)]


class AdjConfig(C.Structure):
    _fields_ = [("LX", C.c_int), ("LY", C.c_int), ("LZ", C.c_int), ("dpd", DpdParams), ("kBT", C.c_float),
                ("mass", C.c_float), ("dt", C.c_float), ("bodyf", C.c_float * 3)]


# name -> (restype, argtypes); every symbol include/ctc_b200.h declares
SIGNATURES = {
    "ctc_status_string": (C.c_char_p, [C.c_int]),
    "ctc_last_error": (C.c_char_p, []),
    "ctc_device_error": (C.c_int, [ip]),
    "ctc_version": (C.c_char_p, []),
    "ctc_dpd_sigma": (C.c_float, [C.c_float, C.c_float, C.c_float]),
    "ctc_rnd_mean0var1": (C.c_int, [C.c_int, C.c_float, vp, vp, C.c_int, vp, vp]),
    "ctc_pair_force": (C.c_int, [C.c_int, C.POINTER(DpdParams), vp, vp, vp, vp, vp]),
    "ctc_clist_ini": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(vp)]),
    "ctc_clist_fin": (C.c_int, [vp]),
    "ctc_clist_build": (C.c_int, [vp, C.c_int, vp, vp, ip, vp]),
    "ctc_clist_get": (C.c_int, [vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp)]),
    "ctc_clist_build_noalloc": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, vp, vp, vp, vp, vp, vp]),
    "ctc_fluforces_ini": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(vp)]),
    "ctc_fluforces_fin": (C.c_int, [vp]),
    "ctc_fluforces_bulk_apply": (C.c_int, [vp, C.POINTER(DpdParams), C.c_int, vp, vp, vp, vp, vp]),
    "ctc_fluforces_halo_apply": (C.c_int, [vp, C.POINTER(DpdParams), C.c_int, vp, vp, vp, vp, vp]),
    "ctc_fluforces_apply_seeded": (C.c_int, [vp, C.POINTER(DpdParams), C.c_int, vp, vp, vp, fp, C.c_int,
                                             C.c_int, vp, vp]),
    "ctc_fluforces_halo_frags": (C.c_int, [vp, vp, ip, vp, vp, vp, vp, vp, vp]),
    "ctc_fluforces_halo_frags_seeded": (C.c_int, [vp, vp, ip, vp, vp, vp, vp, fp, vp, vp]),
    "ctc_fluforces_set_cart": (C.c_int, [vp, ip, ip, C.c_int, ip]),
    "ctc_rbc_force_ini": (C.c_int, [C.c_int, C.c_int, vp, C.c_int, C.POINTER(vp)]),
    "ctc_rbc_force_fin": (C.c_int, [vp]),
    "ctc_rbc_force_md": (C.c_int, [vp, ip]),
    "ctc_rbc_force_set_bending": (C.c_int, [vp, C.c_int]),
    "ctc_rbc_force_apply": (C.c_int, [vp, C.POINTER(RbcParams), C.c_float, C.c_int, vp, vp, vp]),
    "ctc_rbc_area_volume": (C.c_int, [vp, C.c_int, vp, vp, vp]),
    "ctc_cnt_ini": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(vp)]),
    "ctc_cnt_fin": (C.c_int, [vp]),
    "ctc_cnt_apply": (C.c_int, [vp, C.POINTER(DpdLjParams), C.c_int, vp, vp, vp]),
    "ctc_cnt_apply_seeded": (C.c_int, [vp, C.POINTER(DpdLjParams), C.c_int, vp, C.c_float, C.c_float, vp, vp]),
    "ctc_sim_set_contact": (C.c_int, [vp, C.POINTER(DpdLjParams)]),
    "ctc_sim_set_graph": (C.c_int, [vp, C.c_int]),
    "ctc_sim_set_fused_count": (C.c_int, [vp, C.c_int]),
    "ctc_mesh_write_ply": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, vp, vp, C.c_int, C.c_int, C.c_int,
                                     C.c_int]),
    "ctc_sim_set_membrane_noise": (C.c_int, [vp, C.c_int, C.c_uint]),
    "ctc_sim_set_bending": (C.c_int, [vp, C.c_int]),
    "ctc_sim_set_walls": (C.c_int, [vp, vp, C.POINTER(Wvel), C.c_float, vp]),
    "ctc_sim_membrane_count": (C.c_int, [vp, ip, ip]),
    "ctc_sdf_who_stays": (C.c_int, [vp, C.c_int, C.c_int, vp, ip, ip]),
    "ctc_sim_set_walls_strt": (C.c_int, [vp, vp, C.c_char_p, C.POINTER(Wvel), C.c_float]),
    "ctc_sim_wall_strt_dump_templ": (C.c_int, [vp, C.c_char_p]),
    "ctc_wall_strt_dump_templ": (C.c_int, [vp, C.c_char_p]),
    "ctc_wall_strt_ini": (C.c_int, [vp, C.c_char_p, C.POINTER(vp)]),
    "ctc_wall_ini_particles": (C.c_int, [vp, C.c_int, vp, C.POINTER(vp)]),
    "ctc_bop_write": (C.c_int, [C.c_char_p, C.c_long, C.c_int, C.c_char_p, vp]),
    "ctc_bop_read": (C.c_int, [C.c_char_p, C.c_long, C.POINTER(C.c_long), ip, ip, vp]),
    "ctc_restart_write_pp": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int, C.c_long, vp]),
    "ctc_restart_write_ii": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int, C.c_long, vp]),
    "ctc_restart_read_pp": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int, C.c_long, C.POINTER(C.c_long), vp]),
    "ctc_restart_read_ii": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int, C.c_long, C.POINTER(C.c_long), vp]),
    "ctc_io_bop_parts": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int, C.c_long, vp, vp, C.c_int, C.c_int, C.c_int]),
    "ctc_io_bop_ints": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int, C.c_long, vp, C.c_int]),
    "ctc_sdf_ini": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, C.POINTER(vp)]),
    "ctc_sdf_ini_grid": (C.c_int, [C.c_int] * 3 + [vp, vp] + [C.c_int] * 3 + [C.POINTER(vp)]),
    "ctc_sdf_fin": (C.c_int, [vp]),
    "ctc_sdf_read": (C.c_int, [C.c_char_p, ip, vp, vp]),
    "ctc_sdf_resample": (C.c_int, [C.c_int] * 3 + [vp, vp] + [C.c_int] * 3 + [ip, vp, vp, vp, vp]),
    "ctc_sdf_texture": (C.c_int, [vp, ip, vp, vp, vp, vp]),
    "ctc_sdf_eval": (C.c_int, [vp, C.c_int, vp, vp, vp]),
    "ctc_sdf_label": (C.c_int, [vp, C.c_int, vp, vp, vp]),
    "ctc_wall_ini": (C.c_int, [vp, C.c_int, vp, ip, C.POINTER(vp)]),
    "ctc_wall_fin": (C.c_int, [vp]),
    "ctc_wall_particles": (C.c_int, [vp, ip, vp, vp]),
    "ctc_wall_set_vel": (C.c_int, [vp, C.POINTER(Wvel)]),
    "ctc_wall_update_vel": (C.c_int, [vp, C.c_float]),
    "ctc_wall_force": (C.c_int, [vp, C.POINTER(DpdParams), C.c_int, vp, vp, vp]),
    "ctc_wall_force_seeded": (C.c_int, [vp, C.POINTER(DpdParams), C.c_int, vp, C.c_float, vp, vp]),
    "ctc_wall_bounce": (C.c_int, [vp, C.c_float, C.c_int, vp, vp]),
    "ctc_wall_repulse": (C.c_int, [vp, C.c_float, C.c_int, vp, vp, vp]),
    "ctc_rbc_force_set_rnd": (C.c_int, [vp, C.c_int, C.c_uint]),
    "ctc_sim_tune": (C.c_int, [vp, C.c_int, ip, vp]),
    "ctc_sim_set_tune": (C.c_int, [vp, ip]),
    "ctc_fsi_ini": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(vp)]),
    "ctc_fsi_fin": (C.c_int, [vp]),
    "ctc_fsi_apply": (C.c_int, [vp, C.POINTER(DpdParams), C.c_int, vp, C.c_int, vp, vp, vp, vp, vp, vp]),
    "ctc_fsi_apply_seeded": (C.c_int, [vp, C.POINTER(DpdParams), C.c_int, vp, C.c_int, vp, vp, vp, C.c_float,
                                       C.c_float, C.c_int, vp, vp, vp]),
    "ctc_fsi_pairs": (C.c_int, [vp, vp, C.c_int, vp, C.c_int, vp, vp, vp, C.c_float, vp, vp, vp]),
    "ctc_fsi_next_seed": (C.c_int, [vp, fp]),
    "ctc_fsi_set_rank": (C.c_int, [vp, C.c_int]),
    "ctc_scheme_move_apply": (C.c_int, [C.c_float, C.c_float, C.c_int, vp, vp, vp]),
    "ctc_scheme_move_clear_vel": (C.c_int, [C.c_int, vp, vp]),
    "ctc_bforce_apply_cste": (C.c_int, [C.c_float, fp, C.c_int, vp, vp]),
    "ctc_sim_create": (C.c_int, [C.POINTER(SimConfig), C.POINTER(vp)]),
    "ctc_sim_destroy": (C.c_int, [vp]),
    "ctc_sim_set_solvent": (C.c_int, [vp, C.c_int, vp, vp]),
    "ctc_sim_set_solvent_dev": (C.c_int, [vp, C.c_int, vp, vp]),
    "ctc_sim_step": (C.c_int, [vp, C.c_int, vp]),
    "ctc_sim_set_membranes": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, vp, vp, C.POINTER(RbcParams),
                                        C.POINTER(DpdParams), C.c_float, vp]),
    "ctc_sim_get_membranes": (C.c_int, [vp, vp, vp]),
    "ctc_sim_count": (C.c_int, [vp, ip, vp]),
    "ctc_sim_get_solvent": (C.c_int, [vp, vp, ip, vp]),
    "ctc_sim_diag": (C.c_int, [vp, C.POINTER(C.c_double), vp]),
    "ctc_sim_state": (C.c_int, [vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp), C.POINTER(vp)]),
    "ctc_sim_membrane_state": (C.c_int, [vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp)]),
    "ctc_sim_next_seeds": (C.c_int, [vp, fp]),
    "ctc_sim_profile": (C.c_int, [vp, C.c_int]),
    "ctc_sim_profile_read": (C.c_int, [vp, C.POINTER(C.c_double), ip]),
    "ctc_sub_create": (C.c_int, [C.POINTER(SubConfig), C.POINTER(vp)]),
    "ctc_sub_destroy": (C.c_int, [vp]),
    "ctc_sub_set_solvent": (C.c_int, [vp, C.c_int, vp, vp, C.c_int, vp]),
    "ctc_sub_distr_pack": (C.c_int, [vp, vp]),
    "ctc_sub_distr_counts": (C.c_int, [vp, ip]),
    "ctc_sub_distr_unpack": (C.c_int, [vp, ip, vp]),
    "ctc_sub_exch_pack": (C.c_int, [vp, vp]),
    "ctc_sub_exch_counts": (C.c_int, [vp, ip]),
    "ctc_sub_bulk": (C.c_int, [vp, vp]),
    "ctc_sub_halo_update": (C.c_int, [vp, ip, vp]),
    "ctc_sub_bags": (C.c_int, [vp, C.c_int, C.POINTER(vp), C.POINTER(vp), ip]),
    "ctc_bags_copy": (C.c_int, [C.c_int, C.POINTER(vp), C.POINTER(vp), C.POINTER(C.c_longlong), vp]),
    "ctc_sub_count": (C.c_int, [vp, ip, vp]),
    "ctc_sub_set_membranes": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, vp, vp, vp, C.c_int, C.POINTER(RbcParams),
                                        C.POINTER(DpdParams), C.c_float]),
    "ctc_sub_mem_distr_pack": (C.c_int, [vp, vp]),
    "ctc_sub_mem_distr_counts": (C.c_int, [vp, ip]),
    "ctc_sub_mem_distr_unpack": (C.c_int, [vp, ip, vp]),
    "ctc_sub_mem_exch_pack": (C.c_int, [vp, vp]),
    "ctc_sub_mem_exch_counts": (C.c_int, [vp, ip]),
    "ctc_sub_mem_fsi": (C.c_int, [vp, ip, vp]),
    "ctc_sub_mem_update": (C.c_int, [vp, vp]),
    "ctc_sub_get_membranes": (C.c_int, [vp, ip, ip, vp, vp, vp]),
    "ctc_sub_membrane_state": (C.c_int, [vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp)]),
    "ctc_sub_state": (C.c_int, [vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp), C.POINTER(vp)]),
    "ctc_sub_seeds": (C.c_int, [vp, fp]),
    "ctc_sub_masks": (C.c_int, [vp, C.POINTER(C.c_uint)]),
    "ctc_batch_create": (C.c_int, [C.POINTER(BatchConfig), C.POINTER(vp)]),
    "ctc_batch_destroy": (C.c_int, [vp]),
    "ctc_batch_set_solvent": (C.c_int, [vp, vp, vp]),
    "ctc_batch_set_membranes": (C.c_int, [vp, vp, C.c_int, C.c_int, vp, vp, C.POINTER(RbcParams),
                                          C.POINTER(DpdParams), C.c_float, vp]),
    "ctc_batch_step": (C.c_int, [vp, C.c_int, vp]),
    "ctc_batch_set_graph": (C.c_int, [vp, C.c_int]),
    "ctc_batch_tune": (C.c_int, [vp, C.c_int, ip, vp]),
    "ctc_batch_set_tune": (C.c_int, [vp, ip]),
    "ctc_batch_set_persistent": (C.c_int, [vp, C.c_int]),
    "ctc_batch_persistent_check": (C.c_int, [vp, C.c_int, ip, vp]),
    "ctc_batch_persistent_grid": (C.c_int, [vp, ip]),
    "ctc_batch_persistent_stages": (C.c_int, [vp, C.c_int, C.POINTER(C.c_double), vp]),
    "ctc_batch_get_solvent": (C.c_int, [vp, vp, vp]),
    "ctc_batch_get_membranes": (C.c_int, [vp, vp, vp]),
    "ctc_batch_count": (C.c_int, [vp, ip, ip]),
    "ctc_adj_create": (C.c_int, [C.POINTER(AdjConfig), C.c_int, vp, C.c_int, C.c_int, C.c_int, vp, vp,
                                 C.POINTER(RbcParams), C.POINTER(DpdParams), C.c_float, C.POINTER(vp)]),
    "ctc_adj_destroy": (C.c_int, [vp]),
    "ctc_adj_set_params": (C.c_int, [vp, C.POINTER(C.c_double)]),
    "ctc_adj_set_state": (C.c_int, [vp, vp, vp]),
    "ctc_adj_forward": (C.c_int, [vp, C.c_int, C.c_int, C.POINTER(C.c_double), vp]),
    "ctc_adj_backward": (C.c_int, [vp, C.POINTER(C.c_double), vp, vp, vp, vp, vp]),
    "ctc_adj_backward_cot": (C.c_int, [vp, vp, vp, vp, vp, C.POINTER(C.c_double), vp, vp, vp, vp, vp]),
    "ctc_adj_get_final": (C.c_int, [vp, vp, vp, vp]),
}

_lib = None


class CtcError(RuntimeError):
    pass


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise CtcError("libctc_b200.so is not built (run __graft_entry__.build() or "
                           "python -m ctc_b200.build)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status):
    if status != CTC_OK:
        L = lib()
        raise CtcError("%s: %s" % (L.ctc_status_string(status).decode(), L.ctc_last_error().decode()))


def device_error():
    code = C.c_int(0)
    check(lib().ctc_device_error(C.byref(code)))
    return code.value
