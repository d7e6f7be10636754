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


# ---- membranes, FSI and contact (oracle/refkern/refobj.cu) --------------------
_RBC_FIELDS = ("gammaC", "gammaT", "kBT", "kb", "phi", "ks", "x0", "mpow", "ka", "kd", "kv", "totArea", "totVolume")


def _rbc_par(par):
    import numpy as np
    return np.array([par[k] for k in _RBC_FIELDS], np.float32)


def _osig(L):
    vp, i, f = C.c_void_p, C.c_int, C.c_float
    L.refkern_area_volume.argtypes = [i, i, i, vp, vp, vp]
    L.refkern_rbc_force.argtypes = [vp, f, i, i, i, vp, vp, vp, f, f, vp, vp]
    L.refkern_kantor.argtypes = [vp, i, i, i, vp, vp, vp, vp]
    L.refkern_fsi_bulk.argtypes = [f] * 4 + [i] * 4 + [vp, i, vp, vp, f, vp, vp]
    L.refkern_fsi_halo.argtypes = [f] * 4 + [i] * 3 + [vp, vp, i, vp, vp, f, vp, vp]
    L.refkern_cnt_bulk.argtypes = [vp, i, i, i, i, vp, vp, vp, f, vp]
    L.refkern_cnt_halo.argtypes = [vp, i, i, i, vp, vp, i, vp, vp, vp, f, vp, vp]


def _olib():
    L_ = lib()
    _osig(L_)
    return L_


def _tri4(tri):
    import numpy as np
    tri = np.asarray(tri)[:, :3]
    t4 = np.zeros((len(tri), 4), np.int32)
    t4[:, :3] = tri
    return t4


def area_volume(tri, nv, pp):
    """area_volume_compute of the reference (float, atomics): (nc, 2) float32
    [torch, device] of the cells pp (torch (nc*nv, 6) AoS)."""
    import torch
    t4 = torch.as_tensor(_tri4(tri), device=pp.device)
    nc = int(pp.shape[0]) // nv
    av = torch.zeros(2 * nc, dtype=torch.float32, device=pp.device)
    torch.cuda.synchronize()
    assert _olib().refkern_area_volume(nc, nv, len(t4), _p(pp), _p(t4), _p(av)) == 0
    return av.view(nc, 2)


def stressful(nt, totArea):
    """rbc_force_set_stressful (src/rbc/force/imp/main.h:50-59): a0 = totArea /
    nt in float, l0 = sqrt(4 a0 / sqrt(3)) in double, stored as float."""
    import numpy as np
    a0 = np.float32(np.float32(totArea) / np.float32(nt))
    l0 = np.float32(np.sqrt(np.float64(a0) * 4.0 / np.sqrt(3.0)))
    return float(l0), float(a0)


def rbc_force(par, dt, tri, nv, adj0, adj1, md, pp, av, ff):
    """rbc_force_dev::force (stress-ful, no random force) of the cells pp
    (torch (nc*nv, 6)) with the per-cell av (torch float32 (nc, 2)); adds to ff
    (torch (nc*nv, 3)).  adj0/adj1: the ring tables (torch int32, device)."""
    import torch
    l0, a0 = stressful(len(tri), par["totArea"])
    q = _rbc_par(par)                                   # host: the kernel takes the view by value
    nc = int(pp.shape[0]) // nv
    torch.cuda.synchronize()
    assert _olib().refkern_rbc_force(q.ctypes.data_as(C.c_void_p), float(dt), md, nv, nc, _p(pp), _p(adj0), _p(adj1), l0, a0,
                                     _p(av.contiguous()), _p(ff)) == 0


def kantor(par, nv, adj0, adj1, md, pp, ff):
    """kantor_dev::force of the cells pp; adds to ff."""
    import torch
    q = _rbc_par(par)                                   # host: the kernel takes the view by value
    nc = int(pp.shape[0]) // nv
    torch.cuda.synchronize()
    assert _olib().refkern_kantor(q.ctypes.data_as(C.c_void_p), md, nv, nc, _p(pp), _p(adj0), _p(adj1), _p(ff)) == 0


def fsi_bulk(dpd, L, pv, ps, starts, seed, fv, fs):
    """fsi_dev::bulk: vertices pv against the cell-sorted solvent ps (torch
    AoS) with cell starts; adds to fv and fs."""
    import torch
    torch.cuda.synchronize()
    assert _olib().refkern_fsi_bulk(*[float(x) for x in dpd], *L, int(pv.shape[0]), _p(pv), int(ps.shape[0]),
                                    _p(ps), _p(starts), float(seed), _p(fv), _p(fs)) == 0


def images(L, pv_host):
    """The object halo's image list in receive order (the oracle's restatement
    of src/exch/map/dev.h, ascending vertex order in a fragment): counts per
    fragment, the vertex of each image and the image positions (AoS, shifted by
    -d(fid) L as the exchange unpacks them)."""
    import numpy as np
    from . import fsi_halo_images, frag_dir, frag_anti
    frag, vert = fsi_halo_images(L, pv_host)
    slot = np.array([frag_anti(int(f)) for f in frag], np.int64)
    counts = np.bincount(slot, minlength=26).astype(np.int32) if len(frag) else np.zeros(26, np.int32)
    img = np.array(pv_host, np.float32)[vert].copy()
    dirs = np.array([frag_dir(f) for f in range(26)], np.float32)
    if len(frag):
        img[:, :3] -= dirs[frag] * np.asarray(L, np.float32)
    # images sent in fragment fid arrive in receive slot anti(fid), slot after slot
    assert len(frag) == 0 or np.all(np.diff(slot) >= 0)
    return counts, vert, img


def fsi_halo(dpd, L, pv_host, ps, starts, seed, fv, fs):
    """fsi_dev::halo on the images of the vertices pv_host [host]; the image
    forces go back to their vertices in fv (as eobj unpack_ff); adds to fs."""
    import numpy as np
    import torch
    counts, vert, img = images(L, pv_host)
    if len(vert) == 0:
        return 0
    dev = ps.device
    c26 = np.ascontiguousarray(counts, np.int32)
    pimg = torch.as_tensor(img, device=dev)
    fimg = torch.zeros((len(img), 3), dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    assert _olib().refkern_fsi_halo(*[float(x) for x in dpd], *L, c26.ctypes.data_as(C.c_void_p), _p(pimg),
                                    int(ps.shape[0]), _p(ps), _p(starts), float(seed), _p(fimg), _p(fs)) == 0
    fv.index_add_(0, torch.as_tensor(vert.astype(np.int64), device=dev), fimg)
    return len(vert)


def vertex_cells(L, pv_host):
    """The vertex cell list of cnt_build_cells (project = true): starts (nc+1)
    and ids (the clist map codes, object 0: the vertex index) [host int32]."""
    import numpy as np
    from . import clist_build
    counts, starts, order, _ = clist_build(L, pv_host, project=True)
    return np.ascontiguousarray(starts, np.int32), np.ascontiguousarray(order, np.int32)


def cnt(p, L, pv_host, seed_bulk, seed_halo, fv):
    """cnt_dev::bulk then cnt_dev::halo of one object type on the vertices
    pv_host [host]; adds to fv (torch (nv, 3)), image forces returned to their
    vertices."""
    import numpy as np
    import torch
    dev = fv.device
    starts, ids = vertex_cells(L, pv_host)
    pv = torch.as_tensor(np.ascontiguousarray(pv_host, np.float32), device=dev)
    st, ii = torch.as_tensor(starts, device=dev), torch.as_tensor(ids, device=dev)
    lj = np.ascontiguousarray(p, np.float32)            # host: the kernel takes PairDPDLJ by value
    ljp = lj.ctypes.data_as(C.c_void_p)
    lib_ = _olib()
    torch.cuda.synchronize()
    assert lib_.refkern_cnt_bulk(ljp, *L, int(pv.shape[0]), _p(pv), _p(st), _p(ii), float(seed_bulk), _p(fv)) == 0
    counts, vert, img = images(L, pv_host)
    if len(vert) == 0:
        return
    c26 = np.ascontiguousarray(counts, np.int32)
    pimg = torch.as_tensor(img, device=dev)
    fimg = torch.zeros((len(img), 3), dtype=torch.float32, device=dev)
    assert lib_.refkern_cnt_halo(ljp, *L, c26.ctypes.data_as(C.c_void_p), _p(pimg), int(pv.shape[0]), _p(pv),
                                 _p(st), _p(ii), float(seed_halo), _p(fimg), _p(fv)) == 0
    fv.index_add_(0, torch.as_tensor(vert.astype(np.int64), device=dev), fimg)


# ---- the reference's host membrane pieces (oracle/_ref/librefhost.so) ---------
HOST_PATH = os.path.join(_HERE, "_ref", "librefhost.so")
_hlib = None


def host_available():
    return os.path.exists(HOST_PATH)


def hlib():
    global _hlib
    if _hlib is None:
        L_ = C.CDLL(HOST_PATH)
        vp, i = C.c_void_p, C.c_int
        L_.refhost_adj.argtypes = [i, i, i, vp, vp, vp]
        L_.refhost_kantor.argtypes = [C.c_double, C.c_double, i, i, i, vp, i, vp, vp]
        _hlib = L_
    return _hlib


def host_adj(tri, nv, md):
    """adj_ini of the reference (src/rbc/adj/imp/ini.h): adj0, adj1 [md nv]."""
    import numpy as np
    t4 = _tri4(tri)
    a0 = np.zeros(md * nv, np.int32)
    a1 = np.zeros(md * nv, np.int32)
    assert hlib().refhost_adj(md, len(t4), nv, t4.ctypes.data_as(C.c_void_p), a0.ctypes.data_as(C.c_void_p),
                              a1.ctypes.data_as(C.c_void_p)) == 0
    return a0, a1


def host_kantor(tri, nv, md, pp, kb, phi_deg=0.0):
    """The Kantor forces of the cells pp [host (nc*nv, 6)] from the reference's
    host build of its dihedral forces (FP64): (nc*nv, 3) float64."""
    import numpy as np
    t4 = _tri4(tri)
    pp = np.ascontiguousarray(pp, np.float32)
    ff = np.zeros((len(pp), 3), np.float64)
    assert hlib().refhost_kantor(float(phi_deg), float(kb), md, len(t4), nv, t4.ctypes.data_as(C.c_void_p),
                                 len(pp) // nv, pp.ctypes.data_as(C.c_void_p), ff.ctypes.data_as(C.c_void_p)) == 0
    return ff
