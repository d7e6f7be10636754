"""ctc_b200 -- B200-native per-step particle hot path of uDeviceX (rossinelli/CTC).

The compute path is libctc_b200.so (hand-written sm_100a CUDA behind the C ABI
of include/ctc_b200.h).  This module is the host-side mirror of the
reference's module interface for Python callers and the tests: the same
module and function names (clist_build, fluforces_bulk_apply, ...), the same
argument meaning and the same accumulate-into-forces convention.  Device
arrays are torch CUDA tensors (PyTorch is only the device-memory plumbing);
particle arrays use the reference's AoS layout, shape (n, 6) float32.
"""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import CTC_RNG_REFERENCE, CTC_RNG_STABLE, CtcError, check, device_error, lib

__all__ = ["Clist", "FluForces", "Sim", "Batch", "DpdParams", "DpdLjParams", "RbcParams", "RbcForce", "Fsi", "Contact",
           "dpd_sigma", "mesh_write_ply", "scheme_move_apply",
           "scheme_move_clear_vel", "bforce_apply_cste", "rnd_mean0var1", "CTC_RNG_REFERENCE",
           "CTC_RNG_STABLE", "CtcError", "device_error"]


def _torch():
    import torch
    return torch


def _stream(stream=None):
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def _ptr(t):
    if t is None:
        return None
    if not t.is_cuda or not t.is_contiguous():
        raise CtcError("expected a contiguous CUDA tensor")
    return C.c_void_p(t.data_ptr())


def DpdParams(a, g, s, spow):
    """PairDPD {a, g, s, spow} (src/pair/type.h:7-9)."""
    return _lib.DpdParams(a, g, s, spow)


def DpdLjParams(a, g, s, spow, ljs, lje):
    """PairDPDLJ {a, g, s, spow, ljs, lje} (src/pair/type.h:22-25): DPD plus a
    capped Lennard-Jones repulsion, the membrane-membrane contact pair."""
    return _lib.DpdLjParams(a, g, s, spow, ljs, lje)


def dpd_sigma(kBT, g, dt):
    """sigma = sqrt(2 kBT g / dt) (src/pair/imp/main.h:54-62)."""
    return float(lib().ctc_dpd_sigma(kBT, g, dt))


class Clist:
    """Cell lists of one box (src/clist/imp.h): ``Clist(L, maxp).build(pp)``."""

    def __init__(self, L, maxp):
        self.L = tuple(int(x) for x in L)
        self.h = C.c_void_p()
        check(lib().ctc_clist_ini(*self.L, int(maxp), C.byref(self.h)))

    def __del__(self):
        if getattr(self, "h", None) and self.h.value and _lib._lib is not None:
            lib().ctc_clist_fin(self.h)
            self.h = None

    def build(self, pp, stream=None):
        """clist_build: returns (ppout[nout,6], starts[ncells+1], counts[ncells], ids[nout])."""
        torch = _torch()
        n = int(pp.shape[0])
        out = torch.empty_like(pp)
        nout = C.c_int(0)
        check(lib().ctc_clist_build(self.h, n, _ptr(pp), _ptr(out), C.byref(nout), _stream(stream)))
        s, c, i = C.c_void_p(), C.c_void_p(), C.c_void_p()
        check(lib().ctc_clist_get(self.h, C.byref(s), C.byref(c), C.byref(i)))
        nc = self.L[0] * self.L[1] * self.L[2]
        starts = _wrap_dev(s.value, nc + 1, torch.int32, pp.device).clone()
        counts = _wrap_dev(c.value, nc, torch.int32, pp.device).clone()
        ids = _wrap_dev(i.value, nout.value, torch.int32, pp.device).clone()
        return out[:nout.value], starts, counts, ids


class _DevArray:
    """A raw device address seen through __cuda_array_interface__."""

    def __init__(self, addr, n, typestr):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (addr, False),
                                         "version": 2}


def _wrap_dev(addr, n, dtype, device):
    """Copy n elements at a device address into a new tensor."""
    torch = _torch()
    if n <= 0:
        return torch.empty(0, dtype=dtype, device=device)
    typestr = {torch.int32: "<i4", torch.float32: "<f4"}[dtype]
    return torch.as_tensor(_DevArray(addr, n, typestr), device=device)


class FluForces:
    """Solvent DPD forces of one periodic box (src/fluforces/imp.h).

    Holds the trunk generators like fluforces_bulk_ini / fluforces_halo_ini:
    ``bulk_apply`` and ``halo_apply`` draw their seeds as the reference does;
    ``apply_seeded`` takes explicit seeds (27 floats: bulk, then fragments)."""

    def __init__(self, L, maxp):
        self.L = tuple(int(x) for x in L)
        self.h = C.c_void_p()
        check(lib().ctc_fluforces_ini(*self.L, int(maxp), C.byref(self.h)))

    def __del__(self):
        if getattr(self, "h", None) and self.h.value and _lib._lib is not None:
            lib().ctc_fluforces_fin(self.h)
            self.h = None

    def bulk_apply(self, params, pp, starts, counts, ff, stream=None):
        check(lib().ctc_fluforces_bulk_apply(self.h, C.byref(params), int(pp.shape[0]), _ptr(pp), _ptr(starts),
                                             _ptr(counts), _ptr(ff), _stream(stream)))

    def halo_apply(self, params, pp, starts, counts, ff, stream=None):
        check(lib().ctc_fluforces_halo_apply(self.h, C.byref(params), int(pp.shape[0]), _ptr(pp), _ptr(starts),
                                             _ptr(counts), _ptr(ff), _stream(stream)))

    def apply_seeded(self, params, pp, starts, counts, seeds, ff, which=3, rng=CTC_RNG_REFERENCE, stream=None):
        sd = (C.c_float * 27)(*[float(x) for x in np.asarray(seeds, np.float32).reshape(-1)[:27]])
        check(lib().ctc_fluforces_apply_seeded(self.h, C.byref(params), int(pp.shape[0]), _ptr(pp), _ptr(starts),
                                               _ptr(counts), sd, int(which), int(rng), _ptr(ff), _stream(stream)))

    def set_cart(self, dims, coords, rank, nbr):
        """fluforces_halo_ini's per-rank set-up (src/fluforces/imp/ini.h:22-59):
        the fragment trunks and key masks of the rank at coords of a periodic
        dims cart whose neighbour in direction f is rank nbr[f]."""
        check(lib().ctc_fluforces_set_cart(self.h, (C.c_int * 3)(*dims), (C.c_int * 3)(*coords), int(rank),
                                           (C.c_int * 26)(*nbr)))

    def halo_frags(self, params, lpp, lii, rpp, rstart, ff, seeds26=None, stream=None):
        """fluforces_halo_prepare + _apply on exchanged fragments: lists of 26
        device tensors -- local fragment particles lpp[f] (n, 6), their indices
        lii[f] into ff, remote fragment particles rpp[f] (m, 6) and its cell
        starts rstart[f]; seeds26 None draws the module's trunks."""
        def ptrs(ts):
            return (C.c_void_p * 26)(*[t.data_ptr() if t is not None and t.numel() else None for t in ts])
        ln = (C.c_int * 26)(*[int(t.shape[0]) for t in lpp])
        keep = (ptrs(lpp), ptrs(lii), ptrs(rpp), ptrs(rstart))
        if seeds26 is None:
            check(lib().ctc_fluforces_halo_frags(self.h, C.byref(params), ln, *keep, _ptr(ff), _stream(stream)))
        else:
            sd = (C.c_float * 26)(*[float(x) for x in np.asarray(seeds26, np.float32).reshape(-1)[:26]])
            check(lib().ctc_fluforces_halo_frags_seeded(self.h, C.byref(params), ln, *keep, sd, _ptr(ff),
                                                        _stream(stream)))


def RbcParams(**kw):
    """RbcParams_v (src/rbc/params/imp.h:3-9) from keyword fields."""
    return _lib.RbcParams(**kw)


class RbcForce:
    """Membrane internal forces of cells of one template (src/rbc/force/imp.h)."""

    def __init__(self, tri, nv, max_cells):
        tri = np.ascontiguousarray(tri, np.int32).reshape(-1, 3)
        self.nv, self.nt = int(nv), len(tri)
        self.h = C.c_void_p()
        check(lib().ctc_rbc_force_ini(self.nv, self.nt, tri.ctypes.data_as(C.c_void_p), int(max_cells),
                                      C.byref(self.h)))
        md = C.c_int(0)
        check(lib().ctc_rbc_force_md(self.h, C.byref(md)))
        self.md = md.value

    def __del__(self):
        if getattr(self, "h", None) and self.h.value and _lib._lib is not None:
            lib().ctc_rbc_force_fin(self.h)
            self.h = None

    def set_rnd(self, enable=True, seed=0):
        """rbc_force_set_rnd1: the membrane random force (counter-based normals)."""
        check(lib().ctc_rbc_force_set_rnd(self.h, int(bool(enable)), int(seed) & 0xffffffff))

    BENDING = {"none": 0, "kantor": 1, "juelicher": 2}

    def set_bending(self, kantor=True):
        """rbc_force_set_bending: "kantor" (or True), "none" (or False) or
        "juelicher" (src/rbc/force/bending/juelicher, kb = 1, H0 = -1/2)."""
        mode = self.BENDING[kantor] if isinstance(kantor, str) else int(bool(kantor))
        check(lib().ctc_rbc_force_set_bending(self.h, mode))

    def apply(self, params, pp, ff, dt=5e-4, stream=None):
        """rbc_force_apply: adds the internal forces of pp (nc*nv, 6) to ff (nc*nv, 3)."""
        nc = int(pp.shape[0]) // self.nv
        check(lib().ctc_rbc_force_apply(self.h, C.byref(params), float(dt), nc, _ptr(pp), _ptr(ff),
                                        _stream(stream)))

    def area_volume(self, pp, stream=None):
        torch = _torch()
        nc = int(pp.shape[0]) // self.nv
        av = torch.empty((nc, 2), dtype=torch.float64, device=pp.device)
        check(lib().ctc_rbc_area_volume(self.h, nc, _ptr(pp), _ptr(av), _stream(stream)))
        return av


class Fsi:
    """Solvent-membrane DPD forces of one periodic box (src/fsi/imp.h)."""

    def __init__(self, L, maxv, maxs):
        self.h = C.c_void_p()
        check(lib().ctc_fsi_ini(*(int(x) for x in L), int(maxv), int(maxs), C.byref(self.h)))

    def __del__(self):
        if getattr(self, "h", None) and self.h.value and _lib._lib is not None:
            lib().ctc_fsi_fin(self.h)
            self.h = None

    def apply(self, params, pv, ps, starts, counts, fv, fs, stream=None):
        check(lib().ctc_fsi_apply(self.h, C.byref(params), int(pv.shape[0]), _ptr(pv), int(ps.shape[0]), _ptr(ps),
                                  _ptr(starts), _ptr(counts), _ptr(fv), _ptr(fs), _stream(stream)))

    def apply_seeded(self, params, pv, ps, starts, counts, seed_bulk, seed_halo, fv, fs, rng=CTC_RNG_REFERENCE,
                     stream=None):
        check(lib().ctc_fsi_apply_seeded(self.h, C.byref(params), int(pv.shape[0]), _ptr(pv), int(ps.shape[0]),
                                         _ptr(ps), _ptr(starts), _ptr(counts), float(seed_bulk), float(seed_halo),
                                         int(rng), _ptr(fv), _ptr(fs), _stream(stream)))

    def pairs(self, params, pv, ps, starts, counts, seed, fv, fs, stream=None):
        """fsi_bulk of the vertices pv, or fsi_halo of the images pv listed by
        the object exchange: the cells of the box only, keys (seed, index in pv,
        solvent index)."""
        check(lib().ctc_fsi_pairs(self.h, C.byref(params), int(pv.shape[0]), _ptr(pv), int(ps.shape[0]), _ptr(ps),
                                  _ptr(starts), _ptr(counts) if counts is not None else None, float(seed), _ptr(fv),
                                  _ptr(fs), _stream(stream)))

    def next_seed(self):
        s = C.c_float(0)
        check(lib().ctc_fsi_next_seed(self.h, C.byref(s)))
        return s.value


class Contact:
    """Membrane-membrane contact forces of one object type in a periodic box
    (src/cnt/imp.h: cnt_build_cells + cnt_bulk + cnt_halo)."""

    def __init__(self, L, maxv):
        self.h = C.c_void_p()
        check(lib().ctc_cnt_ini(*(int(x) for x in L), int(maxv), C.byref(self.h)))

    def __del__(self):
        if getattr(self, "h", None) and self.h.value and _lib._lib is not None:
            lib().ctc_cnt_fin(self.h)
            self.h = None

    def apply(self, params, pv, fv, stream=None):
        """Draws the bulk and halo seeds of the trunk; pv (n, 6) AoS, fv (n, 3) accumulated."""
        check(lib().ctc_cnt_apply(self.h, C.byref(params), int(pv.shape[0]), _ptr(pv), _ptr(fv), _stream(stream)))

    def apply_seeded(self, params, pv, seed_bulk, seed_halo, fv, stream=None):
        check(lib().ctc_cnt_apply_seeded(self.h, C.byref(params), int(pv.shape[0]), _ptr(pv), float(seed_bulk),
                                         float(seed_halo), _ptr(fv), _stream(stream)))


def _vp(a):
    return a.ctypes.data_as(C.c_void_p)


def bop_write(name, data, vars):
    """A bop file name.bop + name.values: data (n, nvars) float32 or int32
    [host], vars the space-separated variable names."""
    data = np.ascontiguousarray(data)
    t = _lib.CTC_BOP_INT if data.dtype.kind in "iu" else _lib.CTC_BOP_FLOAT
    data = np.ascontiguousarray(data, np.int32 if t == _lib.CTC_BOP_INT else np.float32)
    check(lib().ctc_bop_write(str(name).encode(), len(data), t, vars.encode(), _vp(data)))


def bop_read(header):
    """The records of a bop file (header: its .bop path) as an (n, nvars)
    float32 or int32 array; ascii and iascii values files are read too."""
    n, t, nv = C.c_long(), C.c_int(), C.c_int()
    check(lib().ctc_bop_read(str(header).encode(), 0, C.byref(n), C.byref(t), C.byref(nv), None))
    out = np.zeros((n.value, nv.value), np.float32 if t.value == _lib.CTC_BOP_FLOAT else np.int32)
    check(lib().ctc_bop_read(str(header).encode(), out.size, C.byref(n), None, None, _vp(out)))
    return out


def _restart_id(id):
    return {"templ": _lib.CTC_RESTART_TEMPL, "final": _lib.CTC_RESTART_FINAL}.get(id, id)


def restart_write_pp(base, code, id, pp):
    """restart_write_pp (src/io/restart/imp.h): base/code/ID.bop with ID
    "templ", "final" or %05d; pp (n, 6) x y z vx vy vz [host]."""
    pp = np.ascontiguousarray(pp, np.float32).reshape(-1, 6)
    check(lib().ctc_restart_write_pp(str(base).encode(), code.encode(), _restart_id(id), len(pp), _vp(pp)))


def restart_write_ii(base, code, id, ii):
    ii = np.ascontiguousarray(ii, np.int32).reshape(-1)
    check(lib().ctc_restart_write_ii(str(base).encode(), code.encode(), _restart_id(id), len(ii), _vp(ii)))


def _restart_read(fn, base, code, id, shape, dtype):
    n = C.c_long()
    check(fn(str(base).encode(), code.encode(), _restart_id(id), 0, C.byref(n), None))
    out = np.zeros((n.value,) + shape, dtype)
    check(fn(str(base).encode(), code.encode(), _restart_id(id), n.value, C.byref(n), _vp(out)))
    return out


def restart_read_pp(base, code, id):
    return _restart_read(lib().ctc_restart_read_pp, base, code, id, (6,), np.float32)


def restart_read_ii(base, code, id):
    return _restart_read(lib().ctc_restart_read_ii, base, code, id, (), np.int32)


def io_bop_parts(dump_base, name, id, pp, L, ff=None):
    """io_bop_parts / io_bop_parts_forces (src/io/bop/imp.h) of one rank:
    dump_base/bop/name-%05d, positions from the box's edge."""
    pp = np.ascontiguousarray(pp, np.float32).reshape(-1, 6)
    fp = None
    if ff is not None:
        ff = np.ascontiguousarray(ff, np.float32).reshape(-1, 3)
        fp = _vp(ff)
    check(lib().ctc_io_bop_parts(str(dump_base).encode(), name.encode(), int(id), len(pp), _vp(pp), fp,
                                 *(int(x) for x in L)))


def io_bop_ids(dump_base, name, id, ii, colors=False):
    """io_bop_ids (variable "ids") or, colors=True, io_bop_colors ("color")."""
    ii = np.ascontiguousarray(ii, np.int32).reshape(-1)
    check(lib().ctc_io_bop_ints(str(dump_base).encode(), name.encode(), int(id), len(ii), _vp(ii), int(bool(colors))))


def wvel(kind="cste", u=(0.0, 0.0, 0.0), gdot=0.0, vdir=0, gdir=1, half=0, w=0.0, h=1.0):
    """A wall velocity (wvel_set_cste / _shear / _shear_sin / _hs)."""
    t = {"cste": _lib.CTC_WVEL_CSTE, "shear": _lib.CTC_WVEL_SHEAR, "shear_sin": _lib.CTC_WVEL_SHEAR_SIN,
         "hs": _lib.CTC_WVEL_HS}[kind]
    uu = (float(u), 0.0, 0.0) if np.isscalar(u) else tuple(float(x) for x in u)
    return _lib.Wvel(t, (C.c_float * 3)(*uu), float(gdot), int(vdir), int(gdir), int(half), float(w), float(h))


def sdf_read(path):
    """A field file (sdf.dat): grid size N, extents ext and the values (N2, N1, N0)."""
    N = (C.c_int * 3)()
    ext = (C.c_float * 3)()
    check(lib().ctc_sdf_read(str(path).encode(), N, ext, None))
    D = np.zeros((N[2], N[1], N[0]), np.float32)
    check(lib().ctc_sdf_read(str(path).encode(), N, ext, _vp(D)))
    return list(N), list(ext), D


def sdf_resample(N, ext, D, L):
    """Host-only texture build: (T, tex (T2, T1, T0), o, s, threshold)."""
    ext = np.ascontiguousarray(ext, np.float32)
    D = np.ascontiguousarray(D, np.float32)
    T = (C.c_int * 3)()
    check(lib().ctc_sdf_resample(*(int(x) for x in N), _vp(ext), _vp(D), *(int(x) for x in L), T, None, None, None,
                                 None))
    tex = np.zeros((T[2], T[1], T[0]), np.float32)
    o, s, thr = np.zeros(3, np.float32), np.zeros(3, np.float32), np.zeros(1, np.float32)
    check(lib().ctc_sdf_resample(*(int(x) for x in N), _vp(ext), _vp(D), *(int(x) for x in L), T, _vp(o), _vp(s),
                                 _vp(thr), _vp(tex)))
    return list(T), tex, o, s, float(thr[0])


class Sdf:
    """sdf_ini + sdf_gen (src/wall/sdf): a field file path, or (N, ext, D)."""

    def __init__(self, L, path=None, grid=None):
        self.h = C.c_void_p()
        self.L = tuple(int(x) for x in L)
        if path is not None:
            check(lib().ctc_sdf_ini(str(path).encode(), *self.L, C.byref(self.h)))
        else:
            N, ext, D = grid
            ext = np.ascontiguousarray(ext, np.float32)
            D = np.ascontiguousarray(D, np.float32)
            check(lib().ctc_sdf_ini_grid(*(int(x) for x in N), _vp(ext), _vp(D), *self.L, C.byref(self.h)))

    def __del__(self):
        if getattr(self, "h", None) and self.h.value and _lib._lib is not None:
            lib().ctc_sdf_fin(self.h)
            self.h = C.c_void_p()

    def texture(self):
        T = (C.c_int * 3)()
        check(lib().ctc_sdf_texture(self.h, T, None, None, None, None))
        tex = np.zeros((T[2], T[1], T[0]), np.float32)
        o, s, thr = np.zeros(3, np.float32), np.zeros(3, np.float32), np.zeros(1, np.float32)
        check(lib().ctc_sdf_texture(self.h, T, _vp(o), _vp(s), _vp(thr), _vp(tex)))
        return list(T), tex, o, s, float(thr[0])

    def eval(self, pp, out, stream=None):
        check(lib().ctc_sdf_eval(self.h, int(pp.shape[0]), _ptr(pp), _ptr(out), _stream(stream)))

    def label(self, pp, out, stream=None):
        check(lib().ctc_sdf_label(self.h, int(pp.shape[0]), _ptr(pp), _ptr(out), _stream(stream)))

    def who_stays(self, pp, nv):
        """sdf_who_stays: indices of the cells of pp (device (nc*nv, 6)) with
        every vertex in the bulk."""
        nc = int(pp.shape[0]) // int(nv)
        stay = (C.c_int * max(nc, 1))()
        ns = C.c_int(0)
        check(lib().ctc_sdf_who_stays(self.h, nc, int(nv), _ptr(pp), stay, C.byref(ns)))
        return np.array(stay[:ns.value], np.int64)


class Wall:
    """wall_gen_quants + wall_gen_ticket (src/wall): freezes the solvent
    particles pp (host (n, 6)) inside the wall; self.bulk holds the rest."""

    def __init__(self, sdf, pp):
        self.sdf = sdf                 # the field outlives the wall
        self.h = C.c_void_p()
        pp = np.ascontiguousarray(pp, np.float32).reshape(-1, 6).copy()
        n = C.c_int(0)
        check(lib().ctc_wall_ini(sdf.h, len(pp), _vp(pp), C.byref(n), C.byref(self.h)))
        self.bulk = pp[:n.value]

    def __del__(self):
        if getattr(self, "h", None) and self.h.value and _lib._lib is not None:
            lib().ctc_wall_fin(self.h)
            self.h = C.c_void_p()

    def particles(self):
        n = C.c_int(0)
        check(lib().ctc_wall_particles(self.h, C.byref(n), None, None))
        L = self.sdf.L
        pos = np.zeros((n.value, 4), np.float32)
        st = np.zeros((L[0] + 12) * (L[1] + 12) * (L[2] + 12) + 1, np.int32)
        check(lib().ctc_wall_particles(self.h, C.byref(n), _vp(pos), _vp(st)))
        return pos, st

    def set_vel(self, v):
        check(lib().ctc_wall_set_vel(self.h, C.byref(v)))

    def strt_dump_templ(self, base):
        """wall_strt_dump_templ: base/wall.pp/templ."""
        check(lib().ctc_wall_strt_dump_templ(self.h, str(base).encode()))

    @classmethod
    def from_particles(cls, sdf, pos4):
        """wall_gen_ticket alone: a wall from given particles pos4 (host (n, 4))."""
        pos4 = np.ascontiguousarray(pos4, np.float32).reshape(-1, 4)
        w = cls.__new__(cls)
        w.sdf, w.h, w.bulk = sdf, C.c_void_p(), None
        check(lib().ctc_wall_ini_particles(sdf.h, len(pos4), _vp(pos4), C.byref(w.h)))
        return w

    @classmethod
    def strt(cls, sdf, base):
        """A wall from the restart template base/wall.pp/templ."""
        w = cls.__new__(cls)
        w.sdf, w.h, w.bulk = sdf, C.c_void_p(), None
        check(lib().ctc_wall_strt_ini(sdf.h, str(base).encode(), C.byref(w.h)))
        return w

    def update_vel(self, t):
        check(lib().ctc_wall_update_vel(self.h, float(t)))

    def force(self, params, pp, ff, seed=None, stream=None):
        if seed is None:
            check(lib().ctc_wall_force(self.h, C.byref(params), int(pp.shape[0]), _ptr(pp), _ptr(ff),
                                       _stream(stream)))
        else:
            check(lib().ctc_wall_force_seeded(self.h, C.byref(params), int(pp.shape[0]), _ptr(pp), float(seed),
                                              _ptr(ff), _stream(stream)))

    def bounce(self, dt, pp, stream=None):
        check(lib().ctc_wall_bounce(self.h, float(dt), int(pp.shape[0]), _ptr(pp), _stream(stream)))

    def repulse(self, lam, pp, ff, stream=None):
        check(lib().ctc_wall_repulse(self.h, float(lam), int(pp.shape[0]), _ptr(pp), _ptr(ff), _stream(stream)))


def mesh_write_ply(path, pv, tri, nv, L, shift="edge"):
    """mesh_write_particles (src/io/mesh/imp/main.h): the membranes pv
    (nc*nv, 6) AoS [host] with the template's triangles tri (nt, 3) as the
    reference's binary PLY; shift "edge" (x + L/2) or "center"."""
    pv = np.ascontiguousarray(pv, np.float32).reshape(-1, 6)
    tri = np.ascontiguousarray(tri, np.int32).reshape(-1, 3)
    check(lib().ctc_mesh_write_ply(str(path).encode(), len(pv) // int(nv), int(nv), len(tri),
                                   tri.ctypes.data_as(C.c_void_p), pv.ctypes.data_as(C.c_void_p),
                                   0 if shift == "edge" else 1, *(int(x) for x in L)))


def scheme_move_apply(dt, mass, ff, pp, stream=None):
    """src/scheme/move/imp.h:5 -- v += f/m dt; r += v dt (in place on pp)."""
    check(lib().ctc_scheme_move_apply(dt, mass, int(pp.shape[0]), _ptr(ff), _ptr(pp), _stream(stream)))


def scheme_move_clear_vel(pp, stream=None):
    check(lib().ctc_scheme_move_clear_vel(int(pp.shape[0]), _ptr(pp), _stream(stream)))


def bforce_apply_cste(mass, a, ff, stream=None):
    av = (C.c_float * 3)(*[float(x) for x in a])
    check(lib().ctc_bforce_apply_cste(mass, av, int(ff.shape[0]), _ptr(ff), _stream(stream)))


def pair_force(params, pa, pb, rnd, stream=None):
    """pair_force<PairDPD> (src/pair/dev.h:111-139) on n pairs of AoS particles."""
    torch = _torch()
    f = torch.empty((pa.shape[0], 3), dtype=torch.float32, device=pa.device)
    check(lib().ctc_pair_force(int(pa.shape[0]), C.byref(params), _ptr(pa), _ptr(pb), _ptr(rnd), _ptr(f),
                               _stream(stream)))
    return f


def rnd_mean0var1(seed, u, v, unsigned=False, stream=None):
    """Pair random numbers rnd::mean0var1ii / mean0var1uu (src/math/rnd/dev.h:57-72)."""
    torch = _torch()
    out = torch.empty(u.shape[0], dtype=torch.float32, device=u.device)
    check(lib().ctc_rnd_mean0var1(int(u.shape[0]), float(seed), _ptr(u), _ptr(v), int(bool(unsigned)),
                                  _ptr(out), _stream(stream)))
    return out


class Sim:
    """Plain DPD solvent in one periodic box on the fast path (cell-sorted
    float4 SoA state on the device, one step = wrap + cell lists, bulk + halo
    DPD, body force, update)."""

    def __init__(self, L, maxp, dpd, mass=1.0, dt=5e-4, bodyf=(0.0, 0.0, 0.0), rng=CTC_RNG_REFERENCE):
        cfg = _lib.SimConfig()
        cfg.LX, cfg.LY, cfg.LZ = (int(x) for x in L)
        cfg.maxp = int(maxp)
        cfg.dpd = dpd
        cfg.mass = mass
        cfg.dt = dt
        cfg.bodyf = (C.c_float * 3)(*bodyf)
        cfg.rng = rng
        self.maxp = int(maxp)
        self.L = tuple(int(x) for x in L)
        self.h = C.c_void_p()
        check(lib().ctc_sim_create(C.byref(cfg), C.byref(self.h)))

    def close(self):
        if getattr(self, "h", None) and self.h.value and _lib._lib is not None:
            lib().ctc_sim_destroy(self.h)
            self.h = None

    __del__ = close

    def set_solvent(self, pp, stream=None):
        pp = np.ascontiguousarray(pp, np.float32).reshape(-1, 6)
        check(lib().ctc_sim_set_solvent(self.h, len(pp), pp.ctypes.data_as(C.c_void_p), _stream(stream)))

    def set_membranes(self, pv, tri, nv, params, fsi, mass=0.5, stream=None):
        """Cells of one template: pv (nc*nv, 6) AoS, tri (nt, 3); params a dict of
        RbcParams fields, fsi a DpdParams."""
        pv = np.ascontiguousarray(pv, np.float32).reshape(-1, 6)
        tri = np.ascontiguousarray(tri, np.int32).reshape(-1, 3)
        self.mnv, self.mnc = int(nv), len(pv) // int(nv)
        check(lib().ctc_sim_set_membranes(self.h, self.mnc, self.mnv, len(tri), tri.ctypes.data_as(C.c_void_p),
                                          pv.ctypes.data_as(C.c_void_p), C.byref(_lib.RbcParams(**params)),
                                          C.byref(fsi), float(mass), _stream(stream)))

    def set_graph(self, enable=True):
        """Replay the step as CUDA graphs (captured on first use)."""
        check(lib().ctc_sim_set_graph(self.h, int(bool(enable))))

    def set_fused_count(self, enable=True):
        """The update counts the next cell-list build's cells (default on)."""
        check(lib().ctc_sim_set_fused_count(self.h, int(bool(enable))))

    def tune(self, reps=3, stream=None):
        """Autotune the pair kernels' launch shapes on the current state (after
        a step); returns (bulk threads, bulk unroll, halo threads, halo unroll,
        bulk staging)."""
        ch = (C.c_int * 5)()
        check(lib().ctc_sim_tune(self.h, int(reps), ch, _stream(stream)))
        return tuple(ch)

    def set_tune(self, choice):
        """Launch shapes of the pair kernels (bulk threads, bulk loads in
        flight, halo threads, halo loads[, bulk staging = 0]), as tune()
        returns them."""
        choice = tuple(int(x) for x in choice) + (0,) * (5 - len(choice))
        ch = (C.c_int * 5)(*choice)
        check(lib().ctc_sim_set_tune(self.h, ch))

    def set_membrane_noise(self, enable=True, seed=0):
        """The membrane random force (rbc_force_set_rnd1) from the next step on."""
        check(lib().ctc_sim_set_membrane_noise(self.h, int(bool(enable)), int(seed) & 0xffffffff))

    def set_walls(self, sdf, v=None, lam=0.0, stream=None):
        """Freezes the current solvent against the field sdf (an Sdf of this
        box) and puts the walls in the step: wall forces on the solvent and
        the membranes, the membranes' repulsion lam, bounce-back; v the wall
        velocity (wvel(...), constant zero by default).  None removes them."""
        if sdf is None:
            check(lib().ctc_sim_set_walls(self.h, None, None, 0.0, _stream(stream)))
            self._sdf = None
            return
        v = v if v is not None else wvel("cste")
        check(lib().ctc_sim_set_walls(self.h, sdf.h, C.byref(v), float(lam), _stream(stream)))
        self._sdf = sdf                  # the field outlives the walls
        nc, nv = C.c_int(0), C.c_int(0)  # membranes inside the wall were removed
        check(lib().ctc_sim_membrane_count(self.h, C.byref(nc), C.byref(nv)))
        if getattr(self, "mnv", 0):
            self.mnc = nc.value

    def set_walls_strt(self, sdf, base, v=None, lam=0.0):
        """Walls from the restart template base/wall.pp/templ (the solvent as it is)."""
        v = v if v is not None else wvel("cste")
        check(lib().ctc_sim_set_walls_strt(self.h, sdf.h, str(base).encode(), C.byref(v), float(lam)))
        self._sdf = sdf

    def wall_strt_dump_templ(self, base):
        """The walls' restart template base/wall.pp/templ."""
        check(lib().ctc_sim_wall_strt_dump_templ(self.h, str(base).encode()))

    def set_bending(self, mode="kantor"):
        """The membranes' bending in the step: "kantor", "juelicher" or "none"
        (set after set_membranes, which starts with "kantor")."""
        check(lib().ctc_sim_set_bending(self.h, RbcForce.BENDING[mode]))

    def set_contact(self, params):
        """Membrane-membrane contact (a DpdLjParams) from the next step on; None: off."""
        check(lib().ctc_sim_set_contact(self.h, None if params is None else C.byref(params)))

    def get_membranes(self, stream=None):
        out = np.zeros((self.mnc * self.mnv, 6), np.float32)
        check(lib().ctc_sim_get_membranes(self.h, out.ctypes.data_as(C.c_void_p), _stream(stream)))
        return out

    def step(self, n=1, stream=None):
        check(lib().ctc_sim_step(self.h, int(n), _stream(stream)))

    def strt_dump(self, base, id, name="rbc"):
        """The restart files of the state (flu_strt_dump and rbc_strt_dump,
        src/flu/imp/start.h, src/rbc/imp/start.h): base/flu.pp/ID and, with
        membranes, base/<name>.pp/ID."""
        restart_write_pp(base, "flu.pp", id, self.get_solvent())
        if getattr(self, "mnv", 0):
            restart_write_pp(base, name + ".pp", id, self.get_membranes())

    def get_solvent(self, stream=None):
        out = np.zeros((self.maxp, 6), np.float32)
        n = C.c_int(0)
        check(lib().ctc_sim_get_solvent(self.h, out.ctypes.data_as(C.c_void_p), C.byref(n), _stream(stream)))
        return out[:n.value]

    def diag(self, stream=None):
        out = (C.c_double * 5)()
        check(lib().ctc_sim_diag(self.h, out, _stream(stream)))
        return np.array(out[:])

    def next_seeds(self):
        s = (C.c_float * 27)()
        check(lib().ctc_sim_next_seeds(self.h, s))
        return np.array(s[:], np.float32)

    def forces(self):
        """Copies of the last step's force arrays: the solvent's (cell-sorted,
        (n, 3)) and the membrane vertices' ((nc*nv, 3), empty without
        membranes), as device tensors."""
        torch = _torch()
        dev = torch.device("cuda", torch.cuda.current_device())
        fp = C.c_void_p()
        check(lib().ctc_sim_state(self.h, None, None, C.byref(fp), None))
        n = int(self.get_count())
        fs = _wrap_dev(fp.value, 4 * n, torch.float32, dev).reshape(n, 4)[:, :3].contiguous()
        nc, nv = C.c_int(0), C.c_int(0)
        check(lib().ctc_sim_membrane_count(self.h, C.byref(nc), C.byref(nv)))
        nvt = nc.value * nv.value
        fv = torch.zeros((0, 3), dtype=torch.float32, device=dev)
        if nvt > 0:
            mp = C.c_void_p()
            check(lib().ctc_sim_membrane_state(self.h, None, None, C.byref(mp)))
            fv = _wrap_dev(mp.value, 4 * nvt, torch.float32, dev).reshape(nvt, 4)[:, :3].contiguous()
        return fs, fv

    def get_count(self):
        """Solvent particles in the box (device count of the last build)."""
        st = C.c_void_p()
        check(lib().ctc_sim_state(self.h, None, None, None, C.byref(st)))
        torch = _torch()
        dev = torch.device("cuda", torch.cuda.current_device())
        nc = self.L[0] * self.L[1] * self.L[2]
        return int(_wrap_dev(st.value + 4 * nc, 1, torch.int32, dev).item())

    def profile(self, enable=True):
        """Record per-phase CUDA events on every following step."""
        check(lib().ctc_sim_profile(self.h, int(bool(enable))))

    def profile_read(self):
        """Mean device milliseconds per step of each phase since profile(),
        as {phase name: ms}, and the number of steps; restarts the count."""
        ms = (C.c_double * _lib.CTC_SIM_PHASES)()
        n = C.c_int(0)
        check(lib().ctc_sim_profile_read(self.h, ms, C.byref(n)))
        k = max(n.value, 1)
        return {nm: ms[i] / k for i, nm in enumerate(_lib.SIM_PHASE_NAMES)}, n.value


class Batch:
    """Many independent periodic boxes advanced together: every kernel stage
    of a step is one launch over all boxes; each box is the system a Sim of
    its size would be (its own trunks, box-local RNG keys).  L is a list of
    box sizes, n the solvent particles per box."""

    def __init__(self, L, n, dpd, mass=1.0, dt=5e-4, bodyf=(0.0, 0.0, 0.0), rng=CTC_RNG_REFERENCE):
        self.L = np.ascontiguousarray(np.asarray(L, np.int32).reshape(-1, 3))
        self.n = np.ascontiguousarray(np.asarray(n, np.int32).reshape(-1))
        if len(self.L) != len(self.n):
            raise CtcError("one particle count per box")
        cfg = _lib.BatchConfig()
        cfg.nbox = len(self.n)
        cfg.L = self.L.ctypes.data_as(C.POINTER(C.c_int))
        cfg.n = self.n.ctypes.data_as(C.POINTER(C.c_int))
        cfg.dpd = dpd
        cfg.mass = mass
        cfg.dt = dt
        cfg.bodyf = (C.c_float * 3)(*bodyf)
        cfg.rng = rng
        self.h = C.c_void_p()
        self.mnv, self.nvt = 0, 0
        check(lib().ctc_batch_create(C.byref(cfg), C.byref(self.h)))

    def close(self):
        if getattr(self, "h", None) and self.h.value and _lib._lib is not None:
            lib().ctc_batch_destroy(self.h)
            self.h = None

    __del__ = close

    def set_solvent(self, pp, stream=None):
        """pp (sum n, 6) float32 AoS, box after box."""
        pp = np.ascontiguousarray(pp, np.float32).reshape(-1, 6)
        if len(pp) != int(self.n.sum()):
            raise CtcError("expected %d particles" % int(self.n.sum()))
        check(lib().ctc_batch_set_solvent(self.h, pp.ctypes.data_as(C.c_void_p), _stream(stream)))

    def set_membranes(self, cells, pv, tri, nv, params, fsi, mass=0.5, stream=None):
        """cells[k] membranes in box k; pv (sum cells * nv, 6) AoS box after box."""
        cells = np.ascontiguousarray(np.asarray(cells, np.int32).reshape(-1))
        pv = np.ascontiguousarray(pv, np.float32).reshape(-1, 6)
        tri = np.ascontiguousarray(tri, np.int32).reshape(-1, 3)
        check(lib().ctc_batch_set_membranes(self.h, cells.ctypes.data_as(C.c_void_p), int(nv), len(tri),
                                            tri.ctypes.data_as(C.c_void_p), pv.ctypes.data_as(C.c_void_p),
                                            C.byref(_lib.RbcParams(**params)), C.byref(fsi), float(mass),
                                            _stream(stream)))
        self.mnv, self.nvt = int(nv), len(pv)

    def step(self, n=1, stream=None):
        check(lib().ctc_batch_step(self.h, int(n), _stream(stream)))

    def set_graph(self, enable=True):
        check(lib().ctc_batch_set_graph(self.h, int(bool(enable))))

    def set_persistent(self, enable=True):
        """Each step as one persistent cooperative launch (grid-wide barriers
        between its stages) instead of one launch per stage; enable = 2, 3 or
        4 takes the kernel built for that many blocks per SM (128, 80 or 64
        registers; True: 4, the fastest measured)."""
        check(lib().ctc_batch_set_persistent(self.h, int(enable)))

    def persistent_check(self, barrier, stream=None):
        """One persistent step in which block 0 never arrives at `barrier`:
        returns the launch's blocks; the device error word then holds
        CTC_DEV_WAIT_TIMEOUT (the state is undefined)."""
        blocks = C.c_int(0)
        check(lib().ctc_batch_persistent_check(self.h, int(barrier), C.byref(blocks), _stream(stream)))
        return blocks.value

    def persistent_grid(self):
        blocks = C.c_int(0)
        check(lib().ctc_batch_persistent_grid(self.h, C.byref(blocks)))
        return blocks.value

    def persistent_stages(self, enable=True, stream=None):
        """Record (enable) the persistent step's per-stage times; returns the
        last step's 12 stage times and their sum (ms) when recording was on."""
        ms = (C.c_double * 13)()
        check(lib().ctc_batch_persistent_stages(self.h, int(bool(enable)), ms, _stream(stream)))
        return list(ms)

    def tune(self, reps=3, stream=None):
        """Autotune the pair kernels' launch shapes on the current state;
        returns (bulk threads, bulk unroll, halo threads, halo unroll)."""
        ch = (C.c_int * 4)()
        check(lib().ctc_batch_tune(self.h, int(reps), ch, _stream(stream)))
        return tuple(ch)

    def set_tune(self, choice):
        """(bulk threads, bulk unroll, halo threads[, halo unroll = 2])."""
        choice = tuple(choice) + (2,) * (4 - len(choice))
        ch = (C.c_int * 4)(*choice)
        check(lib().ctc_batch_set_tune(self.h, ch))

    def get_solvent(self, stream=None):
        out = np.zeros((int(self.n.sum()), 6), np.float32)
        check(lib().ctc_batch_get_solvent(self.h, out.ctypes.data_as(C.c_void_p), _stream(stream)))
        return out

    def get_membranes(self, stream=None):
        out = np.zeros((self.nvt, 6), np.float32)
        if self.nvt:
            check(lib().ctc_batch_get_membranes(self.h, out.ctypes.data_as(C.c_void_p), _stream(stream)))
        return out
