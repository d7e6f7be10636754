"""ctypes front end of oracle/_ref/librefkern.so: the reference's own device
code (src/math/rnd/dev.h, src/pair/dev.h, the fluforces and Juelicher
kernels) built from its sources by
oracle/ref.mk.  TEST INFRASTRUCTURE ONLY.  Arrays are torch CUDA tensors."""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
PATH = os.path.join(_HERE, "_ref", "librefkern.so")
_lib = None


def available():
    return os.path.exists(PATH)


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(PATH)
        vp = C.c_void_p
        L.refkern_rnd.argtypes = [C.c_int, C.c_float, vp, vp, C.c_int, vp]
        L.refkern_pair.argtypes = [C.c_int] + [C.c_float] * 4 + [vp, vp, vp, vp]
        _lib = L
    return _lib


def _p(t):
    return C.c_void_p(t.data_ptr())


def rnd(seed, u, v, unsigned=False):
    import torch
    out = torch.empty(u.shape[0], dtype=torch.float32, device=u.device)
    torch.cuda.synchronize()
    assert lib().refkern_rnd(int(u.shape[0]), float(seed), _p(u), _p(v), int(unsigned), _p(out)) == 0
    return out


def pair(dpd, pa, pb, r):
    import torch
    f = torch.empty((pa.shape[0], 3), dtype=torch.float32, device=pa.device)
    torch.cuda.synchronize()
    assert lib().refkern_pair(int(pa.shape[0]), *[float(x) for x in dpd], _p(pa), _p(pb), _p(r), _p(f)) == 0
    return f


def _sig(L):
    vp = C.c_void_p
    L.refkern_bulk.argtypes = [C.c_float] * 4 + [C.c_int] * 4 + [vp, vp, C.c_float, vp]
    L.refkern_halo.argtypes = [C.c_float] * 4 + [C.c_int] * 5 + [vp, vp, vp, vp, C.c_float, C.c_int, vp]


def bulk(dpd, L, pp, starts, seed, ff):
    """fluforces bulk: adds the reference kernel's forces to ff (torch, (n,3))."""
    import torch
    lib_ = lib()
    _sig(lib_)
    torch.cuda.synchronize()
    assert lib_.refkern_bulk(*[float(x) for x in dpd], *L, int(pp.shape[0]), _p(pp), _p(starts), float(seed),
                             _p(ff)) == 0


def fragments(L, starts, counts):
    """Packed fragment lists of src/exch/flu/dev/{map,pack}.h: for every
    fragment the sorted indices of its particles (fragment cells x-fastest)
    and the fragment-cell starts (ncells + 1)."""
    import numpy as np
    from . import frag_dir
    L = tuple(int(x) for x in L)
    out = []
    for fid in range(26):
        d = frag_dir(fid)
        org = [L[c] - 1 if d[c] == 1 else 0 for c in range(3)]
        ext = [L[c] if d[c] == 0 else 1 for c in range(3)]
        z, y, x = np.meshgrid(np.arange(ext[2]), np.arange(ext[1]), np.arange(ext[0]), indexing="ij")
        cid = ((org[0] + x) + L[0] * ((org[1] + y) + L[1] * (org[2] + z))).reshape(-1)
        cnt = counts[cid]
        fss = np.zeros(len(cid) + 1, np.int32)
        fss[1:] = np.cumsum(cnt)
        ii = np.concatenate([np.arange(starts[c], starts[c] + counts[c]) for c in cid]).astype(np.int32) \
            if fss[-1] > 0 else np.zeros(0, np.int32)
        out.append((ii, fss))
    return out


def halo(dpd, L, pp, starts, counts, seeds26, ff):
    """fluforces halo of a 1-rank periodic box with the reference kernel: for
    fragment fid the local list is fragment fid, the remote one its
    anti-fragment (what the self-neighbour sends back), ff accumulated."""
    import numpy as np
    import torch
    from . import frag_anti, halo_masks
    lib_ = lib()
    _sig(lib_)
    starts_h = starts.cpu().numpy() if hasattr(starts, "cpu") else np.asarray(starts)
    counts_h = counts.cpu().numpy() if hasattr(counts, "cpu") else np.asarray(counts)
    fr = fragments(L, starts_h, counts_h)
    masks = halo_masks()
    dev = pp.device
    packed = []
    for ii, fss in fr:
        idx = torch.as_tensor(ii.astype(np.int64), device=dev)
        packed.append((pp[idx].contiguous(), torch.as_tensor(ii, device=dev), torch.as_tensor(fss, device=dev)))
    torch.cuda.synchronize()
    for fid in range(26):
        lpp, lii, _ = packed[fid]
        rpp, _, rss = packed[frag_anti(fid)]
        n = int(lii.shape[0])
        if n == 0:
            continue
        rp = rpp if rpp.shape[0] > 0 else torch.zeros((1, 6), device=dev)
        assert lib_.refkern_halo(*[float(x) for x in dpd], *L, fid, n, _p(lpp), _p(lii), _p(rp), _p(rss),
                                 float(seeds26[fid]), int(masks[fid]), _p(ff)) == 0


def dihedrals(tri):
    """One (i, j, k, l) per edge j-k as juelicher_ini lists them
    (src/rbc/force/bending/juelicher/imp/main.h:46-52): i the third vertex of
    the triangle of the half-edge j -> k, l that of k -> j (taken from the
    j < k side; the dihedral angle and its derivatives are the same from
    either side)."""
    import numpy as np
    tri = np.asarray(tri)[:, :3]
    third = {}
    for a, b, c in tri:
        third[(a, b)], third[(b, c)], third[(c, a)] = c, a, b
    return np.array([(i, j, k, third[(k, j)]) for (j, k), i in third.items() if j < k], np.int32)


def juelicher(tri, nv, pp, ff):
    """juelicher_apply's kernels on the cells pp (torch (nc*nv, 6) AoS); adds
    their forces to ff (torch, (nc*nv, 3))."""
    import numpy as np
    import torch
    tri = np.asarray(tri)[:, :3]
    t4 = torch.zeros((len(tri), 4), dtype=torch.int32)
    t4[:, :3] = torch.as_tensor(tri.astype(np.int32))
    d4 = torch.as_tensor(dihedrals(tri))
    t4, d4 = t4.to(pp.device), d4.to(pp.device)
    vp = C.c_void_p
    lib_ = lib()
    lib_.refkern_juelicher.argtypes = [C.c_int] * 4 + [vp, vp, vp, vp]
    torch.cuda.synchronize()
    assert lib_.refkern_juelicher(int(pp.shape[0]) // nv, nv, len(t4), len(d4), _p(pp), _p(t4), _p(d4), _p(ff)) == 0


# ---- walls (oracle/refkern/refwall.cu) -------------------------------------
class RefWvel(C.Structure):
    _fields_ = [("type", C.c_int), ("u", C.c_float * 3), ("gdot", C.c_float), ("vdir", C.c_int),
                ("gdir", C.c_int), ("half", C.c_int), ("h", C.c_float)]


def _wsig(L):
    vp = C.c_void_p
    L.refwall_sdf.restype = vp
    L.refwall_sdf.argtypes = [C.c_int] * 3 + [vp, vp, vp, C.c_float]
    L.refwall_sdf_fin.argtypes = [vp]
    L.refwall_eval.argtypes = [vp, C.c_int, vp, vp]
    L.refwall_label.argtypes = [vp, C.c_int, vp, vp]
    L.refwall_force.argtypes = [vp] + [C.c_int] * 3 + [vp, vp, C.c_int, C.c_int, RefWvel] + [C.c_float] * 5 + \
        [C.c_int, vp, vp]
    L.refwall_bounce.argtypes = [vp] + [C.c_int] * 3 + [RefWvel, C.c_float, C.c_int, vp]
    L.refwall_repulse.argtypes = [vp, C.c_float, C.c_int, vp, vp]


class RefSdf:
    """The reference's field on a 3D texture: tex (T2, T1, T0) float32 [host]."""

    def __init__(self, tex, o, s, thr):
        import numpy as np
        self.lib = lib()
        _wsig(self.lib)
        tex = np.ascontiguousarray(tex, np.float32)
        o, s = np.ascontiguousarray(o, np.float32), np.ascontiguousarray(s, np.float32)
        T2, T1, T0 = tex.shape
        self.h = self.lib.refwall_sdf(T0, T1, T2, tex.ctypes.data_as(C.c_void_p), o.ctypes.data_as(C.c_void_p),
                                      s.ctypes.data_as(C.c_void_p), float(thr))
        assert self.h

    def close(self):
        if self.h:
            self.lib.refwall_sdf_fin(self.h)
            self.h = None

    def eval(self, pp, out):
        import torch
        torch.cuda.synchronize()
        assert self.lib.refwall_eval(self.h, int(pp.shape[0]), _p(pp), _p(out)) == 0

    def label(self, pp, out):
        import torch
        torch.cuda.synchronize()
        assert self.lib.refwall_label(self.h, int(pp.shape[0]), _p(pp), _p(out)) == 0

    def force(self, L, wpos, wstart, wv, dpd, seed, pp, ff):
        import torch
        torch.cuda.synchronize()
        assert self.lib.refwall_force(self.h, *L, _p(wpos), _p(wstart), int(wpos.shape[0]), int(wstart.shape[0]) - 1,
                                      wv, *[float(x) for x in dpd], float(seed), int(pp.shape[0]), _p(pp),
                                      _p(ff)) == 0

    def bounce(self, L, wv, dt, pp):
        import torch
        torch.cuda.synchronize()
        assert self.lib.refwall_bounce(self.h, *L, wv, float(dt), int(pp.shape[0]), _p(pp)) == 0

    def repulse(self, lam, pp, ff):
        import torch
        torch.cuda.synchronize()
        assert self.lib.refwall_repulse(self.h, float(lam), int(pp.shape[0]), _p(pp), _p(ff)) == 0
