"""ctypes front end of the CPU oracle (TEST INFRASTRUCTURE ONLY).

The oracle restates the reference's per-step particle hot path in plain C
(``ctc_oracle.c``).  Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU
baseline leg of ``bench.py`` use it -- as the checker, never as the product.

Particle arrays are the reference's AoS layout ``Particle {float r[3], v[3]}``
(src/inc/type.h:6-8) as numpy ``float32`` arrays of shape ``(n, 6)``.
"""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libctc_oracle.so")
_lib = None

f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")


class Dpd(C.Structure):
    """``PairDPD {a, g, s, spow}`` (src/pair/type.h:7-9)."""
    _fields_ = [("a", C.c_float), ("g", C.c_float), ("s", C.c_float), ("spow", C.c_float)]


class DpdLj(C.Structure):
    """``PairDPDLJ {a, g, s, spow, ljs, lje}`` (src/pair/type.h:22-25)."""
    _fields_ = [("a", C.c_float), ("g", C.c_float), ("s", C.c_float), ("spow", C.c_float),
                ("ljs", C.c_float), ("lje", C.c_float)]


class RbcParams(C.Structure):
    """``RbcParams_v`` (src/rbc/params/imp.h:3-9)."""
    _fields_ = [(k, C.c_float) for k in
                ("gammaC", "gammaT", "kBT", "kb", "phi", "ks", "x0", "mpow", "ka", "kd", "kv",
                 "totArea", "totVolume")]


class Wvel(C.Structure):
    """The wall velocity of one step: type 0 constant u, 1 shear (gdot, vdir,
    gdir, half), 2 Hele-Shaw (u[0], h)."""
    _fields_ = [("type", C.c_int), ("u", C.c_float * 3), ("gdot", C.c_float), ("vdir", C.c_int),
                ("gdir", C.c_int), ("half", C.c_int), ("h", C.c_float)]


def build():
    """Compile the oracle with its Makefile (gcc, OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        sig = {
            "orc_kiss_ini": (None, [u32p, C.c_int, C.c_int, C.c_int, C.c_int]),
            "orc_kiss_get": (C.c_float, [u32p]),
            "orc_mean0var1ii": (C.c_float, [C.c_float, C.c_int, C.c_int]),
            "orc_mean0var1uu": (C.c_float, [C.c_float, C.c_uint32, C.c_uint32]),
            "orc_set_rng_contraction": (None, [C.c_int]),
            "orc_get_rng_contraction": (C.c_int, []),
            "orc_pair_force": (None, [C.c_float] * 4 + [f32p, f32p, C.c_float, f32p]),
            "orc_mean0var1_batch": (None, [C.c_int, C.c_float, i32p, i32p, C.c_int, f32p]),
            "orc_clist_build": (C.c_int, [C.c_int] * 4 + [f32p, C.c_int, i32p, i32p, i32p, f32p]),
            "orc_dpd_bulk": (None, [C.c_int] * 4 + [f32p, i32p, Dpd, C.c_float, f32p]),
            "orc_dpd_bulk_f64": (None, [C.c_int] * 4 + [f32p, i32p, Dpd, C.c_float, f64p]),
            "orc_dpd_bulk_parallel": (None, [C.c_int] * 4 + [f32p, i32p, Dpd, C.c_float, f32p]),
            "orc_dpd_halo": (None, [C.c_int] * 4 + [f32p, i32p, i32p, Dpd, f32p, f32p]),
            "orc_dpd_halo_f64": (None, [C.c_int] * 4 + [f32p, i32p, i32p, Dpd, f32p, f64p]),
            "orc_halo_masks": (None, [i32p]),
            "orc_halo_trunk_ini": (None, [C.c_int, u32p]),
            "orc_frag_i2d": (C.c_int, [C.c_int, C.c_int]),
            "orc_frag_d2i": (C.c_int, [C.c_int, C.c_int, C.c_int]),
            "orc_frag_anti": (C.c_int, [C.c_int]),
            "orc_fsi_bulk": (None, [C.c_int] * 4 + [f32p, C.c_int, f32p, i32p, Dpd, C.c_float, f32p, f32p]),
            "orc_fsi_halo": (None, [C.c_int] * 4 + [f32p, C.c_int, f32p, i32p, Dpd, C.c_float, f32p, f32p]),
            "orc_fsi_halo_images": (C.c_int, [C.c_int] * 4 + [f32p, C.c_void_p, C.c_void_p]),
            "orc_pair_force_dpdlj": (None, [DpdLj, f32p, f32p, C.c_float, f32p]),
            "orc_juelicher_forces": (None, [C.c_int, C.c_int, C.c_int, i32p, f32p, f64p]),
            "orc_cnt_forces": (None, [C.c_int] * 4 + [f32p, DpdLj, C.c_float, C.c_float, f32p]),
            "orc_mesh_md": (C.c_int, [C.c_int, C.c_int, i32p]),
            "orc_adj_build": (C.c_int, [C.c_int] * 3 + [i32p, i32p, i32p]),
            "orc_area_volume": (None, [C.c_int] * 3 + [i32p, f32p, f64p]),
            "orc_area_volume_f32": (None, [C.c_int] * 3 + [i32p, f32p, f32p]),
            "orc_rbc_forces": (None, [C.c_int] * 5 + [i32p, i32p, f32p, f64p, RbcParams, f32p]),
            "orc_rbc_forces_f64": (None, [C.c_int] * 4 + [i32p, i32p, f32p, f64p, RbcParams, f64p]),
            "orc_area_volume_d": (None, [C.c_int] * 3 + [i32p, f64p, f64p]),
            "orc_rbc_forces_d": (None, [C.c_int] * 4 + [i32p, i32p, f64p, f64p, RbcParams, f64p]),
            "orc_rollout_forces_d": (None, [C.c_int] * 4 + [f64p, i32p, f64p, C.c_float, C.c_int, f64p, f64p,
                                                            C.c_float] + [C.c_int] * 4
                                     + [i32p, i32p, i32p, RbcParams, f64p, f64p]),
            "orc_kantor_energy": (C.c_double, [C.c_int, C.c_int, i32p, i32p, f32p, C.c_double, C.c_double]),
            "orc_kantor_vertex_energy": (None, [C.c_int, C.c_int, i32p, i32p, f32p, C.c_double, C.c_double, f64p]),
            "orc_move": (None, [C.c_float, C.c_float, C.c_int, f32p, f32p]),
            "orc_body_force": (None, [C.c_float, f32p, C.c_int, f32p]),
            "orc_wrap": (None, [C.c_int] * 4 + [f32p]),
            "orc_rbc_wrap": (None, [C.c_int] * 5 + [f32p]),
            "orc_diag": (None, [C.c_int, f32p, C.c_double, f64p]),
            "orc_read_floats": (C.c_int, [C.c_char_p, f32p, C.c_int]),
            "orc_num_threads": (C.c_int, []),
            "orc_set_num_threads": (None, [C.c_int]),
            "orc_dpd_step": (C.c_int, [C.c_int] * 4 + [f32p, f32p, Dpd, f32p, C.c_float, C.c_void_p, C.c_float]),
            "orc_sdf_tex_size": (None, [i32p, i32p]),
            "orc_sdf_resample": (None, [i32p, f32p, f32p, i32p, i32p, f32p, f32p, f32p, f32p]),
            "orc_sdf_eval": (None, [f32p, i32p, f32p, f32p, C.c_float, C.c_int, f32p, f32p]),
            "orc_wall_freeze": (C.c_int, [f32p, i32p, f32p, f32p, C.c_float, i32p, C.c_int, f32p, f32p, i32p,
                                          i32p]),
            "orc_wall_force": (None, [f32p, i32p, f32p, f32p, C.c_float, i32p, f32p, i32p, C.c_int, Wvel]
                               + [C.c_float] * 5 + [C.c_int, f32p, f32p]),
            "orc_wall_bounce": (None, [f32p, i32p, f32p, f32p, C.c_float, Wvel, C.c_float, C.c_int, f32p]),
            "orc_wall_repulse": (None, [f32p, i32p, f32p, f32p, C.c_float, C.c_float, C.c_int, f32p, f32p]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _pp(pp):
    return np.ascontiguousarray(pp, dtype=np.float32).reshape(-1, 6)


# ---- RNG -------------------------------------------------------------------
class Kiss:
    """KISS trunk generator (src/math/rnd/imp.cpp:12-34)."""

    def __init__(self, x, y, z, c):
        self.st = np.zeros(4, np.uint32)
        lib().orc_kiss_ini(self.st, x, y, z, c)

    @classmethod
    def halo(cls, fid):
        k = cls(0, 0, 0, 0)
        lib().orc_halo_trunk_ini(fid, k.st)
        return k

    def get(self):
        return float(np.float32(lib().orc_kiss_get(self.st)))


def mean0var1ii(seed, u, v):
    return np.float32(lib().orc_mean0var1ii(seed, int(u), int(v)))


def mean0var1_batch(seed, u, v, unsigned=False):
    u = np.ascontiguousarray(u, np.int32)
    v = np.ascontiguousarray(v, np.int32)
    out = np.zeros(len(u), np.float32)
    lib().orc_mean0var1_batch(len(u), seed, u, v, int(unsigned), out)
    return out


def mean0var1uu(seed, u, v):
    return np.float32(lib().orc_mean0var1uu(seed, int(u), int(v)))


def halo_masks():
    m = np.zeros(26, np.int32)
    lib().orc_halo_masks(m)
    return m


def frag_anti(i):
    return lib().orc_frag_anti(i)


def frag_dir(i):
    return tuple(lib().orc_frag_i2d(i, c) for c in range(3))


# ---- cell lists ------------------------------------------------------------
def clist_build(L, pp, project=False):
    """Returns (counts, starts[ncells+1], order, ppout) -- stable cell order."""
    pp = _pp(pp)
    LX, LY, LZ = L
    nc = LX * LY * LZ
    counts = np.zeros(nc, np.int32)
    starts = np.zeros(nc + 1, np.int32)
    order = np.zeros(max(len(pp), 1), np.int32)
    out = np.zeros((max(len(pp), 1), 6), np.float32)
    nout = lib().orc_clist_build(LX, LY, LZ, len(pp), pp, int(project), counts, starts, order, out)
    starts[nc] = nout
    return counts, starts, order[:nout], out[:nout]


# ---- solvent forces ----------------------------------------------------------
def dpd_bulk(L, pp, starts, dpd, seed, f64=False):
    pp = _pp(pp)
    if f64:
        ff = np.zeros((len(pp), 3), np.float64)
        lib().orc_dpd_bulk_f64(*L, len(pp), pp, starts, Dpd(*dpd), seed, ff)
    else:
        ff = np.zeros((len(pp), 3), np.float32)
        lib().orc_dpd_bulk(*L, len(pp), pp, starts, Dpd(*dpd), seed, ff)
    return ff


def dpd_halo(L, pp, starts, counts, dpd, seeds, f64=False):
    pp = _pp(pp)
    seeds = np.ascontiguousarray(seeds, np.float32)
    if f64:
        ff = np.zeros((len(pp), 3), np.float64)
        lib().orc_dpd_halo_f64(*L, len(pp), pp, starts, counts, Dpd(*dpd), seeds, ff)
    else:
        ff = np.zeros((len(pp), 3), np.float32)
        lib().orc_dpd_halo(*L, len(pp), pp, starts, counts, Dpd(*dpd), seeds, ff)
    return ff


def pair_force(dpd, pa, pb, rnd):
    f = np.zeros(3, np.float32)
    lib().orc_pair_force(*[float(x) for x in dpd], np.asarray(pa, np.float32),
                         np.asarray(pb, np.float32), float(rnd), f)
    return f


# ---- Juelicher bending (src/rbc/force/bending/juelicher) -------------------
def juelicher_forces(tri, nv, pv):
    """The Juelicher bending forces (kb = 1, H0 = -1/2 as the reference
    hard-codes them) of the cells pv (nc*nv, 6) AoS, in double."""
    pv = _pp(pv)
    tri = np.ascontiguousarray(np.asarray(tri, np.int32)[:, :3])
    nc = len(pv) // nv
    ff = np.zeros((len(pv), 3), np.float64)
    lib().orc_juelicher_forces(nc, nv, len(tri), tri, pv, ff)
    return ff


# ---- membrane-membrane contact (src/cnt) -------------------------------------
def pair_force_dpdlj(p, pa, pb, rnd):
    """DPD + Lennard-Jones pair force (src/pair/dev.h:49-75); p = (a, g, s, spow, ljs, lje)."""
    f = np.zeros(3, np.float32)
    lib().orc_pair_force_dpdlj(DpdLj(*p), np.ascontiguousarray(pa, np.float32), np.ascontiguousarray(pb, np.float32),
                               float(rnd), f)
    return f


def cnt_forces(L, pv, p, seed_bulk, seed_halo):
    """Contact forces of one object type (src/cnt bulk + halo) on the vertices
    pv (AoS); p = (a, g, s, spow, ljs, lje)."""
    pv = _pp(pv)
    fv = np.zeros((len(pv), 3), np.float32)
    lib().orc_cnt_forces(*L, len(pv), pv, DpdLj(*p), float(seed_bulk), float(seed_halo), fv)
    return fv


# ---- FSI -------------------------------------------------------------------
def fsi_forces(L, pv, ps, starts, dpd, seed_bulk, seed_halo):
    pv, ps = _pp(pv), _pp(ps)
    fv = np.zeros((len(pv), 3), np.float32)
    fs = np.zeros((len(ps), 3), np.float32)
    lib().orc_fsi_bulk(*L, len(pv), pv, len(ps), ps, starts, Dpd(*dpd), seed_bulk, fv, fs)
    lib().orc_fsi_halo(*L, len(pv), pv, len(ps), ps, starts, Dpd(*dpd), seed_halo, fv, fs)
    return fv, fs


def fsi_halo_images(L, pv):
    pv = _pp(pv)
    n = lib().orc_fsi_halo_images(*L, len(pv), pv, None, None)
    frag = np.zeros(max(n, 1), np.int32)
    vert = np.zeros(max(n, 1), np.int32)
    lib().orc_fsi_halo_images(*L, len(pv), pv, frag.ctypes.data, vert.ctypes.data)
    return frag[:n], vert[:n]


# ---- membrane ----------------------------------------------------------------
def mesh_md(tri, nv):
    tri4 = _tri4(tri)
    return lib().orc_mesh_md(nv, len(tri4), tri4)


def _tri4(tri):
    tri = np.asarray(tri, np.int32)
    if tri.shape[1] == 3:
        tri = np.concatenate([tri, np.zeros((len(tri), 1), np.int32)], 1)
    return np.ascontiguousarray(tri)


def adj_build(tri, nv, md=None):
    tri4 = _tri4(tri)
    if md is None:
        md = lib().orc_mesh_md(nv, len(tri4), tri4)
    a0 = np.zeros(nv * md, np.int32)
    a1 = np.zeros(nv * md, np.int32)
    if lib().orc_adj_build(md, len(tri4), nv, tri4, a0, a1) != 0:
        raise ValueError("mesh is not a closed manifold of valence <= md")
    return md, a0, a1


def area_volume(tri, nv, pp, f32=False):
    tri4 = _tri4(tri)
    pp = _pp(pp)
    nc = len(pp) // nv
    if f32:
        av = np.zeros(2 * nc, np.float32)
        lib().orc_area_volume_f32(nc, nv, len(tri4), tri4, pp, av)
    else:
        av = np.zeros(2 * nc, np.float64)
        lib().orc_area_volume(nc, nv, len(tri4), tri4, pp, av)
    return av.reshape(nc, 2)


def rbc_forces(tri, nv, pp, params, av=None, mode=0, f64=False, ff=None):
    """Internal membrane forces; params is a dict of RbcParams fields.  With ff
    (float32 (n, 3)) the float path adds them onto a copy of ff, slot by slot,
    as the reference's atomics add them onto the force array it is given."""
    tri4 = _tri4(tri)
    pp = _pp(pp)
    md, a0, a1 = adj_build(tri4, nv)
    nc = len(pp) // nv
    if av is None:
        av = area_volume(tri4, nv, pp)
    av = np.ascontiguousarray(av, np.float64).reshape(-1)
    par = RbcParams(**params)
    if f64:
        ff = np.zeros((len(pp), 3), np.float64)
        lib().orc_rbc_forces_f64(nc, nv, md, len(tri4), a0, a1, pp, av, par, ff)
    else:
        ff = np.zeros((len(pp), 3), np.float32) if ff is None else np.array(ff, np.float32).reshape(-1, 3)
        lib().orc_rbc_forces(mode, nc, nv, md, len(tri4), a0, a1, pp, av, par, ff)
    return ff


def rollout_forces_f64(L, pp, ids, dpd, seed, pv=None, fsi=None, fseed=0.0, tri=None, nv=0, params=None):
    """FP64 forces of one step of the differentiable rollout (stable keys):
    solvent pairs, FSI and membrane forces from double positions; returns
    (F (n, 3), Fv (nvt, 3)).  A test reference for the adjoint's gradients."""
    pp = np.ascontiguousarray(pp, np.float64).reshape(-1, 6)
    ids = np.ascontiguousarray(ids, np.int32)
    F = np.zeros((len(pp), 3))
    if pv is None:
        pv, nc, md, a0, a1, tri4 = np.zeros((0, 6)), 0, 0, np.zeros(1, np.int32), np.zeros(1, np.int32), \
            np.zeros(4, np.int32)
        fsi, params = (0.0, 0.0, 0.0, 1.0), dict(gammaC=0, gammaT=0, kBT=0, kb=0, phi=0, ks=0, x0=0.5, mpow=2,
                                                  ka=0, kd=0, kv=0, totArea=1, totVolume=1)
        ntri = 0
    else:
        pv = np.ascontiguousarray(pv, np.float64).reshape(-1, 6)
        tri4 = _tri4(tri)
        md, a0, a1 = adj_build(tri4, nv)
        nc, ntri = len(pv) // nv, len(tri4)
    Fv = np.zeros((len(pv), 3))
    lib().orc_rollout_forces_d(*L, len(pp), pp, ids, np.asarray(dpd, np.float64), float(seed), len(pv), pv,
                               np.asarray(fsi, np.float64), float(fseed), nc, nv, md, ntri, a0, a1, tri4,
                               RbcParams(**params), F, Fv)
    return F, Fv


def kantor_energy(tri, nv, pp, kb, phi_deg=0.0):
    md, a0, a1 = adj_build(tri, nv)
    return lib().orc_kantor_energy(nv, md, a0, a1, _pp(pp), kb, phi_deg)


def kantor_vertex_energy(tri, nv, pp, kb, phi_deg=0.0):
    """Per vertex, the mean over its edges of kb (1 - cos(theta - phi)) with
    the Kantor force's dihedral angle."""
    md, a0, a1 = adj_build(tri, nv)
    ev = np.zeros(nv, np.float64)
    lib().orc_kantor_vertex_energy(nv, md, a0, a1, _pp(pp), kb, phi_deg, ev)
    return ev


# ---- update --------------------------------------------------------------------
def move(pp, ff, dt, mass):
    pp = _pp(pp).copy()
    lib().orc_move(dt, mass, len(pp), np.ascontiguousarray(ff, np.float32), pp)
    return pp


def body_force(ff, mass, a):
    ff = np.ascontiguousarray(ff, np.float32).copy()
    lib().orc_body_force(mass, np.asarray(a, np.float32), len(ff), ff)
    return ff


def wrap(L, pp):
    pp = _pp(pp).copy()
    lib().orc_wrap(*L, len(pp), pp)
    return pp


def rbc_wrap(L, pp, nv):
    pp = _pp(pp).copy()
    lib().orc_rbc_wrap(*L, len(pp) // nv, nv, pp)
    return pp


def diag(pp, mass):
    out = np.zeros(5, np.float64)
    pp = _pp(pp)
    lib().orc_diag(len(pp), pp, mass, out)
    return out


def read_floats(path, cap=1 << 24):
    buf = np.zeros(cap, np.float32)
    n = lib().orc_read_floats(path.encode(), buf, cap)
    if n < 0:
        raise FileNotFoundError(path)
    return buf[:n].copy()


def num_threads():
    return lib().orc_num_threads()


def set_num_threads(n):
    lib().orc_set_num_threads(int(n))


def dpd_step(L, pp, dpd, seeds, mass, bodyf, dt):
    """One plain DPD step in the reference's order (OpenMP)."""
    pp = _pp(pp).copy()
    work = np.zeros_like(pp)
    seeds = np.ascontiguousarray(seeds, np.float32)
    bf = None if bodyf is None else np.ascontiguousarray(bodyf, np.float32)
    n = lib().orc_dpd_step(*L, len(pp), pp, work, Dpd(*dpd), seeds, mass,
                           None if bf is None else bf.ctypes.data, dt)
    return pp[:n]


def _sig_late():
    L = lib()
    if not getattr(L, "_late_sig", False):
        L.orc_wrap_flag.argtypes = [C.c_int] * 4 + [f32p, np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")]
        L.orc_wrap_flag.restype = None
        L.orc_clist_build_late.argtypes = [C.c_int] * 4 + [f32p, C.c_int,
                                                           np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS"),
                                                           i32p, i32p, i32p, f32p]
        L.orc_clist_build_late.restype = C.c_int
        L._late_sig = True
    return L


def distribute(L, pp):
    """Periodic wrap + cell-list rebuild of one step (src/sim/imp/distr.h:14-55):
    particles that re-entered follow the others inside their cell.  Returns
    (counts, starts[ncells+1], ppout)."""
    Lb = _sig_late()
    pp = _pp(pp).copy()
    moved = np.zeros(len(pp), np.uint8)
    Lb.orc_wrap_flag(*L, len(pp), pp, moved)
    nc = L[0] * L[1] * L[2]
    counts = np.zeros(nc, np.int32)
    starts = np.zeros(nc + 1, np.int32)
    order = np.zeros(max(len(pp), 1), np.int32)
    out = np.zeros((max(len(pp), 1), 6), np.float32)
    nout = Lb.orc_clist_build_late(*L, len(pp), pp, 0, moved, counts, starts, order, out)
    starts[nc] = nout
    return counts, starts, out[:nout]


def rbc_step(L, ps, pv, tri, nv, dpd, fsi, rbcpar, seeds27, fsi_seeds, bodyf, dt, ms, mv, cnt=None,
             cnt_seeds=None, bending="kantor"):
    """One step of solvent + membranes in the reference's order
    (src/sim/imp/run.h:8-68), with membrane-membrane contact (cnt: a PairDPDLJ
    tuple, cnt_seeds: its bulk and halo seeds) among the object forces
    (src/sim/objinter/imp/main.h:42-92) and the membranes' bending "kantor"
    or "juelicher" (src/rbc/force/bending/imp.cpp); returns (solvent sorted,
    vertices)."""
    counts, starts, ps = distribute(L, ps)
    pv = rbc_wrap(L, pv, nv)
    fs = dpd_bulk(L, ps, starts, dpd, seeds27[0]) + dpd_halo(L, ps, starts, counts, dpd, seeds27[1:])
    fv, fs2 = fsi_forces(L, pv, ps, starts, fsi, fsi_seeds[0], fsi_seeds[1])
    if cnt is not None:
        fv = fv + cnt_forces(L, pv, cnt, cnt_seeds[0], cnt_seeds[1])
    fs = fs + fs2
    a = np.asarray(bodyf if bodyf is not None else (0, 0, 0), np.float32)
    fs = body_force(fs, ms, a)
    fv = body_force(fv, mv, a)
    ps = move(ps, fs, dt, ms)
    # bending first, then the triangle forces, onto the forces already there
    # (src/sim/objects/imp/main.h:40-48, src/rbc/force/imp/forces.h:53)
    if bending == "juelicher":
        fv = fv + juelicher_forces(tri, nv, pv).astype(np.float32)   # the double sum rounded, then added
        fv = rbc_forces(tri, nv, pv, dict(rbcpar, kb=0.0), mode=0, ff=fv)
    else:
        fv = rbc_forces(tri, nv, pv, rbcpar, mode=0, ff=fv)
    pv = move(pv, fv, dt, mv)
    return ps, pv


# ---- walls (src/wall) --------------------------------------------------------
def sdf_read(path):
    """The sdf.dat field: (N, ext, D (N2, N1, N0) float32)."""
    with open(path, "rb") as f:
        ext = [float(x) for x in f.readline().split()]
        N = [int(x) for x in f.readline().split()]
        D = np.frombuffer(f.read(4 * N[0] * N[1] * N[2]), np.float32).reshape(N[2], N[1], N[0])
    return N, ext, D


class Sdf:
    """The field of one periodic box L on the reference's texture grid
    (sdf_gen, src/wall/sdf/imp/gen.h) and the wall operations on it."""

    def __init__(self, N, ext, D, L):
        self.L = np.asarray(L, np.int32)
        self.T = np.zeros(3, np.int32)
        lib().orc_sdf_tex_size(self.L, self.T)
        self.tex = np.zeros(int(np.prod(self.T)), np.float32)
        self.o, self.s, self.thr = np.zeros(3, np.float32), np.zeros(3, np.float32), np.zeros(1, np.float32)
        lib().orc_sdf_resample(np.asarray(N, np.int32), np.asarray(ext, np.float32),
                               np.ascontiguousarray(D, np.float32).reshape(-1), self.L, self.T, self.tex,
                               self.o, self.s, self.thr)

    def _a(self):
        return self.tex, self.T, self.o, self.s, float(self.thr[0])

    def eval(self, pp):
        pp = _pp(pp)
        out = np.zeros(len(pp), np.float32)
        lib().orc_sdf_eval(*self._a(), len(pp), pp, out)
        return out

    def freeze(self, pp):
        """(bulk particles, wall positions (n, 4) cell-sorted, cell starts)."""
        pp = _pp(pp).copy()
        wpos = np.zeros((27 * max(len(pp), 1), 4), np.float32)
        nc = int(np.prod(self.L + 12))
        ws = np.zeros(nc + 1, np.int32)
        nw = np.zeros(1, np.int32)
        k = lib().orc_wall_freeze(*self._a(), self.L, len(pp), pp, wpos, ws, nw)
        return pp[:k], wpos[:nw[0]], ws

    def force(self, wpos, wstart, wv, dpd, seed, pp):
        pp = _pp(pp)
        ff = np.zeros((len(pp), 3), np.float32)
        lib().orc_wall_force(*self._a(), self.L, np.ascontiguousarray(wpos, np.float32),
                             np.ascontiguousarray(wstart, np.int32), len(wpos), wv, *[float(x) for x in dpd],
                             float(seed), len(pp), pp, ff)
        return ff

    def bounce(self, wv, dt, pp):
        pp = _pp(pp).copy()
        lib().orc_wall_bounce(*self._a(), wv, float(dt), len(pp), pp)
        return pp

    def repulse(self, lam, pp):
        pp = _pp(pp)
        ff = np.zeros((len(pp), 3), np.float32)
        lib().orc_wall_repulse(*self._a(), float(lam), len(pp), pp, ff)
        return ff
