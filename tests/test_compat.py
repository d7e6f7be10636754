"""The C++ compatibility layer (ctc_b200/compat/udx_compat.cpp) defines the
reference's module entry points with the reference's own signatures: the
object compiled against the reference's headers (by __graft_entry__.build()
where the reference tree is present) must export exactly these symbols."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
OBJ = os.path.join(ROOT, "ctc_b200", "compat", "_build", "udx_compat.o")

# the declarations of src/pair/imp.h, src/clist/imp.h, src/fluforces/imp.h
# (bulk and halo), src/fsi/imp.h, src/rbc/force/imp.h,
# src/rbc/force/area_volume/imp.h, src/scheme/force/imp.h,
# src/scheme/move/imp.h, src/io/restart/imp.h and the
# walls' src/wall/imp.h, src/wall/sdf/imp.h, src/wall/wvel/imp.h (the
# MPI_Comm of the compile check is its stand-in type), as the C++ compiler
# names them
EXPECTED = [
    "pair_ini(PairParams**)",
    "pair_fin(PairParams*)",
    "pair_set_dpd(int, float const*, float const*, float, PairParams*)",
    "pair_set_lj(float, float, PairParams*)",
    "pair_set_adhesion(float, float, PairParams*)",
    "pair_set_conf(Config const*, char const*, PairParams*)",
    "pair_compute_dpd_sigma(float, float, PairParams*)",
    "pair_get_view_dpd(PairParams const*, PairDPD*)",
    "pair_get_view_dpd_color(PairParams const*, PairDPDC*)",
    "pair_get_view_dpd_mirrored(PairParams const*, PairDPDCM*)",
    "pair_get_view_dpd_lj(PairParams const*, PairDPDLJ*)",
    "pair_get_view_adhesion(PairParams const*, PairAdhesion*)",
    "fluforces_halo_ini(ctc_compat_check_comm*, int3, FluForcesHalo**)",
    "fluforces_halo_fin(FluForcesHalo*)",
    "fluforces_halo_prepare(Sarray<flu::LFrag, 26>, Sarray<flu::RFrag, 26>, FluForcesHalo*)",
    "fluforces_halo_apply(PairParams const*, FluForcesHalo const*, FoArray const*)",
    "fsi_ini(int, int3, Fsi**)",
    "fsi_fin(Fsi*)",
    "fsi_bind_solvent(PaArray, Force*, int, int const*, Fsi*)",
    "fsi_bulk(Fsi*, int, PairParams const**, PaWrap*, FoWrap*)",
    "fsi_halo(Fsi*, int, PairParams const**, Sarray<Particle*, 26>, Sarray<Force*, 26>, int const*)",
    "area_volume_ini(int, int, int4 const*, int, AreaVolume**)",
    "area_volume_fin(AreaVolume*)",
    "area_volume_compute(AreaVolume*, int, Particle const*, float**)",
    "area_volume_host(AreaVolume*, float**)",
    "bforce_ini(BForce**)",
    "bforce_fin(BForce*)",
    "bforce_set_none(BForce*)",
    "bforce_set_cste(float3, BForce*)",
    "bforce_set_conf(Config const*, BForce*)",
    "bforce_adjust(float3, BForce*)",
    "bforce_apply(Coords const*, float, BForce const*, int, Particle const*, Force*)",
    "clist_ini(int, int, int, Clist**)",
    "clist_fin(Clist*)",
    "clist_ini_map(int, int, Clist const*, ClistMap**)",
    "clist_fin_map(ClistMap*)",
    "clists_get_ss(Clist const*)",
    "clists_get_cc(Clist const*)",
    "clists_get_dim(Clist const*)",
    "clists_get_n(Clist const*)",
    "clist_get_ids(ClistMap const*)",
    "clist_build(int, int, Particle const*, Particle*, Clist*, ClistMap*)",
    "fluforces_bulk_ini(int3, int, FluForcesBulk**)",
    "fluforces_bulk_fin(FluForcesBulk*)",
    "fluforces_bulk_prepare(int, PaArray const*, FluForcesBulk*)",
    "fluforces_bulk_apply(PairParams const*, int, FluForcesBulk const*, int const*, int const*, FoArray const*)",
    "rbc_force_ini(MeshRead const*, RbcForce**)",
    "rbc_force_fin(RbcForce*)",
    "rbc_force_set_stressful(int, float, RbcForce*)",
    "rbc_force_set_rnd0(RbcForce*)",
    "rbc_force_set_rnd1(int, RbcForce*)",
    "rbc_force_set_bending(MeshRead const*, char const*, RbcForce*)",
    "rbc_force_apply(RbcForce*, RbcParams const*, float, RbcQuants const*, Force*)",
    "rbc_force_stat(float*, float*)",
    "rbc_force_set_stressfree(char const*, RbcForce*)",
    "scheme_move_apply(float, float, int, Force const*, Particle*)",
    "scheme_move_clear_vel(int, Particle*)",
    "restart_write_pp(ctc_compat_check_comm*, char const*, char const*, int, long, Particle const*)",
    "restart_write_ii(ctc_compat_check_comm*, char const*, char const*, int, long, int const*)",
    "restart_read_pp(ctc_compat_check_comm*, char const*, char const*, int, int*, Particle*)",
    "restart_read_ii(ctc_compat_check_comm*, char const*, char const*, int, int*, int*)",
    "sdf_ini(int3, Sdf**)",
    "sdf_fin(Sdf*)",
    "sdf_gen(Coords const*, ctc_compat_check_comm*, bool, Sdf*)",
    "sdf_bulk_wall(Sdf const*, int*, Particle*, int*, Particle*)",
    "sdf_who_stays(Sdf const*, int, Particle const*, int, int, int*)",
    "sdf_bounce(float, WvelStep const*, Coords const*, Sdf const*, int, Particle*)",
    "wvel_ini(Wvel**)",
    "wvel_fin(Wvel*)",
    "wvel_step_ini(WvelStep**)",
    "wvel_step_fin(WvelStep*)",
    "wvel_set_cste(float3, Wvel*)",
    "wvel_set_shear(float, int, int, int, Wvel*)",
    "wvel_set_shear_sin(float, int, int, int, float, Wvel*)",
    "wvel_set_hs(float, float, Wvel*)",
    "wvel_get_step(float, Wvel const*, WvelStep*)",
    "wvel_get_type(WvelStep const*)",
    "wall_ini_quants(int3, WallQuants*)",
    "wall_ini_ticket(int3, WallTicket**)",
    "wall_fin_quants(WallQuants*)",
    "wall_fin_ticket(WallTicket*)",
    "wall_gen_quants(ctc_compat_check_comm*, int, int, Sdf const*, int*, Particle*, WallQuants*)",
    "wall_gen_ticket(WallQuants const*, WallTicket*)",
    "wall_strt_quants(ctc_compat_check_comm*, char const*, int, WallQuants*)",
    "wall_strt_dump_templ(ctc_compat_check_comm*, char const*, WallQuants const*)",
    "wall_force(PairParams const*, WvelStep const*, Coords const*, Sdf const*, WallQuants const*, WallTicket const*, "
    "int, PaArray const*, FoArray const*)",
    "wall_repulse(Sdf const*, WallRepulsePrm const*, long, PaArray const*, FoArray const*)",
    "wall_repulse_prm_ini(float, WallRepulsePrm**)",
    "wall_repulse_prm_fin(WallRepulsePrm*)",
]


@pytest.mark.skipif(not os.path.exists(OBJ), reason="compatibility layer not built (needs the reference's headers)")
def test_compat_layer_exports_reference_signatures():
    nm = shutil.which("nm")
    assert nm
    out = subprocess.run([nm, "-C", "--defined-only", OBJ], capture_output=True, text=True, check=True).stdout
    defined = {line.split(" ", 2)[2] for line in out.splitlines() if " T " in line}
    missing = [s for s in EXPECTED if s not in defined]
    assert not missing, missing
