"""Multi-process host logic of the decomposed solvent and membranes (no
GPU): 2, 3, 4 and 8 gloo ranks run the product's step orchestration
(``exch.step``), cart (``exch.Cart``) and transport (``exch.DistTransport``)
over host tensors.  Each rank's subdomain is a numpy stand-in written here --
the same bins, bags, shifts and record layout as the device kernels, with
deterministic DPD forces (no random term) in float64 -- and after three
steps with migration the ranks together hold exactly the undivided periodic
box's state.  With membranes the stand-in also migrates whole cells (binned
by the centre of their bounding box), sends its vertices' images across the
faces for the solvent-vertex forces and takes the images' forces back, as
the device path does; the cells' internal forces are springs.  The device
kernels themselves are tested on the GPU (tests/test_gpu_exch.py)."""
import os
import socket
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
A, G, SPOW, DT = 2.5, 8.0, 0.25, 0.02


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def dpd_forces(pa, va, pb, vb, same):
    """Forces on the particles a from the particles b (float64): conservative
    and dissipative DPD terms; same: a and b are the same set."""
    d = pa[:, None, :] - pb[None, :, :]
    r = np.sqrt((d * d).sum(-1))
    ok = (r < 1.0) & (r > 1e-9)
    if same:
        np.fill_diagonal(ok, False)
    rs = np.where(ok, r, 1.0)
    e = d / rs[..., None]
    w = np.where(ok, (1.0 - rs) ** SPOW, 0.0)
    ev = (e * (va[:, None, :] - vb[None, :, :])).sum(-1)
    mag = np.where(ok, A * (1.0 - rs) - G * w * w * ev, 0.0)
    return (mag[..., None] * e).sum(1)


def pair_matrix(pa, va, pb, vb):
    """Pairwise forces (na, nb, 3) on the particles a from the particles b."""
    d = pa[:, None, :] - pb[None, :, :]
    r = np.sqrt((d * d).sum(-1))
    ok = (r < 1.0) & (r > 1e-9)
    rs = np.where(ok, r, 1.0)
    e = d / rs[..., None]
    w = np.where(ok, (1.0 - rs) ** SPOW, 0.0)
    ev = (e * (va[:, None, :] - vb[None, :, :])).sum(-1)
    mag = np.where(ok, A * (1.0 - rs) - G * w * w * ev, 0.0)
    return mag[..., None] * e


KS, NV = 40.0, 8          # the cells: 8 vertices joined by springs of constant KS


def spring_forces(cr, rest):
    """Internal forces of cells (nc, NV, 3): every vertex pair a spring at its
    rest length."""
    d = cr[:, :, None, :] - cr[:, None, :, :]
    r = np.sqrt((d * d).sum(-1))
    np.einsum("cii->ci", r)[...] = 1.0
    mag = -KS * (r - rest[None])
    np.einsum("cii->ci", mag)[...] = 0.0
    return (mag[..., None] * d / r[..., None]).sum(2)


def undivided_cells(pp, cells, rest, Lg, steps):
    """The periodic box with solvent and cells: solvent pairs and
    solvent-vertex pairs by minimum image, springs inside the cells."""
    r, v = pp[:, :3].copy(), pp[:, 3:].copy()
    cr, cv = cells[..., :3].copy(), cells[..., 3:].copy()
    Lg = np.asarray(Lg, float)
    nc = len(cr)
    for _ in range(steps):
        d = r[:, None, :] - r[None, :, :]
        d -= np.round(d / Lg) * Lg
        img = r[:, None, :] - d
        f = np.zeros_like(r)
        for i in range(len(r)):
            f[i] = dpd_forces(r[i:i + 1], v[i:i + 1], img[i], v, False)[0]
        vr, vv = cr.reshape(-1, 3), cv.reshape(-1, 3)
        dv = vr[:, None, :] - r[None, :, :]
        dv -= np.round(dv / Lg) * Lg                # solvent b's nearest image seen from vertex k
        F = np.zeros((len(vr), len(r), 3))
        for k in range(len(vr)):
            F[k] = pair_matrix(vr[k:k + 1], vv[k:k + 1], vr[k] - dv[k], v)[0]
        fv = F.sum(1).reshape(nc, NV, 3) + spring_forces(cr, rest)
        f -= F.sum(0)
        v = v + f * DT
        r = r + v * DT
        r -= np.floor((r + Lg / 2) / Lg) * Lg
        cv = cv + fv * DT
        cr = cr + cv * DT
    return np.concatenate([r, v], 1), np.concatenate([cr, cv], 2)


def undivided(pp, Lg, steps):
    """The periodic box of edges Lg, all pairs by minimum image."""
    r, v = pp[:, :3].copy(), pp[:, 3:].copy()
    Lg = np.asarray(Lg, float)
    for _ in range(steps):
        d = r[:, None, :] - r[None, :, :]
        d -= np.round(d / Lg) * Lg
        img = r[:, None, :] - d                     # the nearest image of b seen from a
        f = np.zeros_like(r)
        for i in range(len(r)):
            f[i] = dpd_forces(r[i:i + 1], v[i:i + 1], img[i], v, False)[0] - 0.0
        v = v + f * DT
        r = r + v * DT
        r -= np.floor((r + Lg / 2) / Lg) * Lg       # back into [-Lg/2, Lg/2)
    return np.concatenate([r, v], 1)


class NumpySub:
    """A subdomain on the host with the device kernels' bags: records of 8
    floats (x y z id | u v w 0), bins by -1/0/1 per axis, received bag j
    shifted by +d(j) L, halo bag f = the particles of the boundary cells of
    fragment f."""
    REC = 8

    def __init__(self, L, cart, rank, pp, ids):
        from ctc_b200 import exch
        self.X, self.L, self.cart, self.rank = exch, np.array(L), cart, rank
        self.r, self.v, self.ids = pp[:, :3].astype(np.float64), pp[:, 3:].astype(np.float64), ids.copy()
        cap = 4096
        self.send = [torch.zeros(self.REC * cap, dtype=torch.float64) for _ in range(26)]
        self.recv = [torch.zeros(self.REC * cap, dtype=torch.float64) for _ in range(26)]
        self.fsend = [torch.zeros(4, dtype=torch.int32) for _ in range(26)]
        self.frecv = [torch.zeros(4, dtype=torch.int32) for _ in range(26)]

    def _records(self, sel):
        rec = np.zeros((len(sel), 8))
        rec[:, :3], rec[:, 3], rec[:, 4:7] = self.r[sel], self.ids[sel], self.v[sel]
        return rec

    def _bin(self, r):
        lo = -(self.L // 2)
        d = -1 + (r >= lo).astype(int) + (r >= lo + self.L).astype(int)
        return np.array([self.X.frag_d2i(tuple(x)) if any(x) else 26 for x in d], int)

    def distr_pack(self):
        self._dc = self._distr_pack()

    def distr_counts(self):
        return self._dc

    def _distr_pack(self):
        b = self._bin(self.r)
        counts = []
        for f in range(26):
            rec = self._records(np.flatnonzero(b == f))
            self.send[f][:rec.size] = torch.from_numpy(rec.reshape(-1))
            counts.append(len(rec))
        self.bags_counts = counts
        keep = b == 26
        self.r, self.v, self.ids = self.r[keep], self.v[keep], self.ids[keep]
        return counts

    def bags(self, kind, counts):
        if kind == 2:
            return self.fsend, self.frecv, [4] * 26
        return [self.send[f][:self.REC * counts[f]] for f in range(26)], self.recv, [4096] * 26

    def distr_unpack(self, rcounts):
        for j in range(26):
            rec = self.recv[j][:self.REC * rcounts[j]].numpy().reshape(-1, 8)
            r = rec[:, :3] + np.array(self.X.FRAG_DIRS[j]) * self.L
            assert (self._bin(r) == 26).all()
            self.r = np.concatenate([self.r, r])
            self.v = np.concatenate([self.v, rec[:, 4:7]])
            self.ids = np.concatenate([self.ids, rec[:, 3].astype(int)])

    def exch_pack(self):
        self._xc = self._exch_pack()

    def exch_counts(self):
        return self._xc

    def _exch_pack(self):
        lo = -(self.L // 2)
        c = np.floor(self.r - lo).astype(int)
        counts = []
        for f in range(26):
            d = np.array(self.X.FRAG_DIRS[f])
            sel = np.ones(len(c), bool)
            for k in range(3):
                if d[k] == 1:
                    sel &= c[:, k] == self.L[k] - 1
                elif d[k] == -1:
                    sel &= c[:, k] == 0
            rec = self._records(np.flatnonzero(sel))
            self.send[f][:rec.size] = torch.from_numpy(rec.reshape(-1))
            counts.append(len(rec))
        return counts

    def bulk(self):
        self.f = dpd_forces(self.r, self.v, self.r, self.v, True)

    def halo_update(self, rcounts):
        for j in range(26):
            rec = self.recv[j][:self.REC * rcounts[j]].numpy().reshape(-1, 8)
            if len(rec):
                rb = rec[:, :3] + np.array(self.X.FRAG_DIRS[j]) * self.L
                self.f += dpd_forces(self.r, self.v, rb, rec[:, 4:7], False)
        self.v = self.v + self.f * DT
        self.r = self.r + self.v * DT


class NumpySubCells(NumpySub):
    """The stand-in with whole cells of NV vertices: a cell migrates with its
    bounding box's centre (records of NV x 8 floats, vertex id = cell id x NV
    + vertex); a vertex within 1 of a face, or beyond it, sends an image to
    every fragment of those faces; the forces on the images come back in the
    order of the image bags."""

    def __init__(self, L, cart, rank, pp, ids, cells, cell_ids, rest):
        super().__init__(L, cart, rank, pp, ids)
        self.mnv = NV
        self.cr, self.cv = cells[..., :3].astype(np.float64), cells[..., 3:].astype(np.float64)
        self.cids, self.rest = cell_ids.copy(), rest
        ccap, icap = 16, 1024
        z = lambda k: [torch.zeros(k, dtype=torch.float64) for _ in range(26)]
        self.csend, self.crecv = z(self.REC * NV * ccap), z(self.REC * NV * ccap)
        self.isend, self.irecv = z(self.REC * icap), z(self.REC * icap)
        self.bsend, self.brecv = z(4 * icap), z(4 * icap)
        self.caps = {3: ccap, 4: icap, 5: icap}

    def mem_distr_pack(self):
        self._cc = self._mem_distr_pack()

    def mem_distr_counts(self):
        return self._cc

    def _mem_distr_pack(self):
        b = self._bin(0.5 * (self.cr.min(1) + self.cr.max(1)))
        counts = []
        for f in range(26):
            sel = np.flatnonzero(b == f)
            rec = np.zeros((len(sel), NV, 8))
            rec[..., :3], rec[..., 4:7] = self.cr[sel], self.cv[sel]
            rec[..., 3] = self.cids[sel, None] * NV + np.arange(NV)
            self.csend[f][:rec.size] = torch.from_numpy(rec.reshape(-1))
            counts.append(len(sel))
        keep = b == 26
        self.cr, self.cv, self.cids = self.cr[keep], self.cv[keep], self.cids[keep]
        return counts

    def mem_bags(self, kind, counts, rcounts=None):
        if kind == 3:
            return [self.csend[f][:self.REC * NV * counts[f]] for f in range(26)], self.crecv, [self.caps[3]] * 26
        if kind == 4:
            return [self.isend[f][:self.REC * counts[f]] for f in range(26)], self.irecv, [self.caps[4]] * 26
        return [self.bsend[j][:4 * rcounts[j]] for j in range(26)], self.brecv, [self.caps[5]] * 26

    def mem_distr_unpack(self, rcounts):
        for j in range(26):
            rec = self.crecv[j][:self.REC * NV * rcounts[j]].numpy().reshape(-1, NV, 8)
            cr = rec[..., :3] + np.array(self.X.FRAG_DIRS[j]) * self.L
            assert (self._bin(0.5 * (cr.min(1) + cr.max(1))) == 26).all()
            self.cr = np.concatenate([self.cr, cr])
            self.cv = np.concatenate([self.cv, rec[..., 4:7]])
            self.cids = np.concatenate([self.cids, (rec[:, 0, 3] // NV).astype(int)])

    def mem_exch_pack(self):
        self._ic = self._mem_exch_pack()

    def mem_exch_counts(self):
        return self._ic

    def _mem_exch_pack(self):
        lo = -(self.L // 2)
        vr, vv = self.cr.reshape(-1, 3), self.cv.reshape(-1, 3)
        side = np.where(vr < lo + 1, -1, np.where(vr >= lo + self.L - 1, 1, 0))
        sel = [[] for _ in range(26)]
        for i, sd in enumerate(side):
            axes = [k for k in range(3) if sd[k]]
            for m in range(1, 1 << len(axes)):
                d = [0, 0, 0]
                for q, k in enumerate(axes):
                    if (m >> q) & 1:
                        d[k] = int(sd[k])
                sel[self.X.frag_d2i(tuple(d))].append(i)
        self._ivid = [np.array(x, int) for x in sel]
        vid = (self.cids[:, None] * NV + np.arange(NV)).reshape(-1)
        for f in range(26):
            rec = np.zeros((len(sel[f]), 8))
            rec[:, :3], rec[:, 3], rec[:, 4:7] = vr[sel[f]], vid[sel[f]], vv[sel[f]]
            self.isend[f][:rec.size] = torch.from_numpy(rec.reshape(-1))
        return [len(x) for x in sel]

    def mem_fsi(self, rcounts):
        vr, vv = self.cr.reshape(-1, 3), self.cv.reshape(-1, 3)
        F = pair_matrix(vr, vv, self.r, self.v)      # the own vertices, no periodic wrap
        self.mf = F.sum(1)
        self.f -= F.sum(0)
        for j in range(26):
            rec = self.irecv[j][:self.REC * rcounts[j]].numpy().reshape(-1, 8)
            out = np.zeros((len(rec), 4))
            if len(rec):
                Fj = pair_matrix(rec[:, :3] + np.array(self.X.FRAG_DIRS[j]) * self.L, rec[:, 4:7], self.r, self.v)
                self.f -= Fj.sum(0)
                out[:, :3] = Fj.sum(1)
            self.bsend[j][:out.size] = torch.from_numpy(out.reshape(-1))

    def mem_update(self):
        for f in range(26):
            b = self.brecv[f][:4 * len(self._ivid[f])].numpy().reshape(-1, 4)
            np.add.at(self.mf, self._ivid[f], b[:, :3])
        fv = self.mf.reshape(-1, NV, 3) + spring_forces(self.cr, self.rest)
        self.cv = self.cv + fv * DT
        self.cr = self.cr + self.cv * DT


def _rank_main(rank, world, port, dims, L, out, with_cells=False):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import datetime

    import torch.distributed as dist
    from ctc_b200 import exch
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    cart = exch.Cart(dims)
    pp, Lg = _system(dims, L, 2.0 if with_cells else 0.0)
    c = np.floor((pp[:, :3] + np.array(Lg) / 2) / np.array(L)).astype(int)
    me = np.array(cart.coords(rank))
    sel = np.flatnonzero((c == me).all(1))
    o = -np.array(Lg) / 2 + (me + 0.5) * np.array(L)
    q = pp[sel].copy()
    q[:, :3] -= o
    if with_cells:
        cells, rest = _cells(Lg, L)
        cc = 0.5 * (cells[..., :3].min(1) + cells[..., :3].max(1))
        cb = np.floor((cc + np.array(Lg) / 2) / np.array(L)).astype(int)
        csel = np.flatnonzero((cb == me).all(1))
        cq = cells[csel].copy()
        cq[..., :3] -= o
        sub = NumpySubCells(L, cart, rank, q, sel, cq, csel, rest)
    else:
        sub = NumpySub(L, cart, rank, q, sel)
    T = exch.DistTransport(cart, rank)
    for _ in range(3):
        exch.step([sub], T)
    res = np.concatenate([sub.r + o, sub.v], 1)
    cres = (sub.cids.tolist(), np.concatenate([sub.cr + o, sub.cv], 2).tolist()) if with_cells else None
    out.put((rank, sub.ids.tolist(), res.tolist(), cres))
    dist.destroy_process_group()


def _cells(Lg, L):
    """Four cells of NV vertices (a cube of edge 0.7, rotated, perturbed)
    with their springs' rest lengths; two sit just inside a face (the one
    between the first two ranks along x, and the periodic one) and drift
    across it with the solvent."""
    rng = np.random.default_rng(9)
    cube = np.array([[x, y, z] for x in (-0.35, 0.35) for y in (-0.35, 0.35) for z in (-0.35, 0.35)])
    rest = np.sqrt(((cube[:, None] - cube[None]) ** 2).sum(-1))
    hx = Lg[0] / 2
    face = -hx + L[0]                       # between the first two ranks along x
    centres = [(face - 0.02, 0.3, 0.2), (hx - 0.02, -0.9, 0.6), (-hx / 2, Lg[1] / 2 - 0.3, -Lg[2] / 2 + 0.2),
               (hx / 2, 0.4, -0.5)]
    cells = []
    for c in centres:
        q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
        r = cube @ q.T + np.array(c) + rng.normal(0, 0.02, (NV, 3))
        v = rng.normal(0, 0.3, (NV, 3)) + np.array([2.0, 0.0, 0.0])
        cells.append(np.concatenate([r, v], 1))
    return np.array(cells), rest


def _system(dims, L, drift=0.0):
    Lg = tuple(d * l for d, l in zip(dims, L))
    rng = np.random.default_rng(7)
    n = 3 * int(np.prod(Lg))
    r = -np.array(Lg) / 2 + rng.random((n, 3)) * np.array(Lg)
    v = rng.normal(0, 1.5, (n, 3))
    v[:, 0] += drift
    return np.concatenate([r, v], 1), Lg


@pytest.mark.parametrize("dims", [(2, 1, 1), (2, 2, 1), (2, 2, 2)])
def test_ranks_gloo_equal_undivided_box(dims):
    import torch.multiprocessing as mp
    L = (4, 4, 4)
    world = dims[0] * dims[1] * dims[2]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, dims, L, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    pp, Lg = _system(dims, L)
    ref = undivided(pp, Lg, 3)
    got = np.full_like(ref, np.nan)
    seen = np.zeros(len(pp), int)
    for rank, ids, st, _ in res:
        got[ids] = np.array(st).reshape(-1, 6)
        seen[ids] += 1
    assert (seen == 1).all()
    d = got[:, :3] - ref[:, :3]
    d -= np.round(d / np.array(Lg)) * np.array(Lg)
    assert np.abs(d).max() < 1e-9
    assert np.abs(got[:, 3:] - ref[:, 3:]).max() < 1e-9
    # some particles changed rank on the way
    moved = sum(int((np.floor((np.array(st).reshape(-1, 6)[:, :3] + np.array(Lg) / 2) / np.array(L)) !=
                     np.floor((pp[ids, :3] + np.array(Lg) / 2) / np.array(L))).any(1).sum()) for _, ids, st, _ in res)
    assert moved > 0


def _run_ranks(dims, L, with_cells):
    import torch.multiprocessing as mp
    world = dims[0] * dims[1] * dims[2]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, dims, L, q, with_cells)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    return res


@pytest.mark.parametrize("dims", [(3, 1, 1), (2, 1, 1), (2, 2, 1), (2, 2, 2)])
def test_ranks_gloo_cells_equal_undivided_box(dims):
    """Solvent and cells flowing along x: after three steps the ranks hold
    exactly the undivided box's solvent and cells (1e-9), every cell on one
    rank, and the two cells placed just inside a face have changed rank."""
    L = (4, 4, 4)
    res = _run_ranks(dims, L, True)
    pp, Lg = _system(dims, L, 2.0)
    cells, rest = _cells(Lg, L)
    ref, cref = undivided_cells(pp, cells, rest, Lg, 3)
    Lg = np.array(Lg, float)
    got = np.full_like(ref, np.nan)
    cgot = np.full_like(cref, np.nan)
    owner = np.full(len(cells), -1)
    for rank, ids, st, (cids, cst) in res:
        got[ids] = np.array(st).reshape(-1, 6)
        assert (owner[cids] == -1).all()
        owner[cids] = rank
        cgot[cids] = np.array(cst).reshape(-1, NV, 6)
    assert (owner >= 0).all()
    d = got[:, :3] - ref[:, :3]
    d -= np.round(d / Lg) * Lg
    assert np.abs(d).max() < 1e-9 and np.abs(got[:, 3:] - ref[:, 3:]).max() < 1e-9
    d = cgot[..., :3] - cref[..., :3]
    d -= np.round(d / Lg) * Lg
    assert np.abs(d).max() < 1e-9 and np.abs(cgot[..., 3:] - cref[..., 3:]).max() < 1e-9
    from ctc_b200 import exch
    cart = exch.Cart(dims)
    start = np.floor((0.5 * (cells[..., :3].min(1) + cells[..., :3].max(1)) + Lg / 2) / np.array(L)).astype(int)
    first = [cart.rank(tuple(c)) for c in start]
    assert owner[0] != first[0] and owner[1] != first[1], (owner, first)


def test_cart_neighbours_are_symmetric():
    from ctc_b200 import exch
    for dims in [(1, 1, 1), (2, 1, 1), (3, 2, 1), (2, 2, 2), (4, 3, 2)]:
        cart = exch.Cart(dims)
        for r in range(cart.size):
            nb = cart.neighbours(r)
            assert cart.rank(cart.coords(r)) == r
            for f in range(26):
                assert cart.neighbours(nb[f])[exch.frag_anti(f)] == r


# -- ranks of one process: bags moved by address ---------------------------------
class _HostCopies:
    """Stands in for the library's ctc_bags_copy on host memory."""

    def __init__(self):
        self.launches = 0

    def ctc_bags_copy(self, n, dst, src, nbytes, stream):
        import ctypes
        self.launches += 1
        for k in range(n):
            ctypes.memmove(dst[k], src[k], nbytes[k])
        return 0


class PtrSubCells(NumpySubCells):
    """The numpy stand-in with its bags as addresses (SubDomain.bag_ptrs'
    contract: send addresses, units sent, receive addresses, capacities,
    bytes per unit), for LocalTransport.exchange_ptrs."""

    def _stream(self):
        return None

    def bag_ptrs(self, kind, counts, rcounts=None):
        rec = 8 * self.REC
        if kind == 0 or kind == 1:
            return ([t.data_ptr() for t in self.send], counts, [t.data_ptr() for t in self.recv],
                    [4096] * 26, rec)
        if kind == 2:
            return ([t.data_ptr() for t in self.fsend], [4] * 26, [t.data_ptr() for t in self.frecv], [4] * 26, 4)
        if kind == 3:
            return ([t.data_ptr() for t in self.csend], counts, [t.data_ptr() for t in self.crecv],
                    [self.caps[3]] * 26, rec * NV)
        if kind == 4:
            return ([t.data_ptr() for t in self.isend], counts, [t.data_ptr() for t in self.irecv],
                    [self.caps[4]] * 26, rec)
        return ([t.data_ptr() for t in self.bsend], rcounts, [t.data_ptr() for t in self.brecv],
                counts, 32)


@pytest.mark.parametrize("dims", [(3, 1, 1), (2, 1, 1), (2, 2, 1)])
def test_local_transport_by_address_equals_undivided_box(dims, monkeypatch):
    """All ranks in one process (LocalTransport): exch.step moves every bag
    by address, one copy call per exchange, and after three steps of solvent
    and cells flowing across the faces the ranks hold exactly the undivided
    box's state."""
    from ctc_b200 import exch
    fake = _HostCopies()
    monkeypatch.setattr(exch, "lib", lambda: fake)
    L = (4, 4, 4)
    cart = exch.Cart(dims)
    pp, Lg = _system(dims, L, 2.0)
    cells, rest = _cells(Lg, L)
    c = np.floor((pp[:, :3] + np.array(Lg) / 2) / np.array(L)).astype(int)
    cc = 0.5 * (cells[..., :3].min(1) + cells[..., :3].max(1))
    cb = np.floor((cc + np.array(Lg) / 2) / np.array(L)).astype(int)
    subs, origins = [], []
    for r in range(cart.size):
        me = np.array(cart.coords(r))
        o = -np.array(Lg) / 2 + (me + 0.5) * np.array(L)
        sel = np.flatnonzero((c == me).all(1))
        q = pp[sel].copy()
        q[:, :3] -= o
        csel = np.flatnonzero((cb == me).all(1))
        cq = cells[csel].copy()
        cq[..., :3] -= o
        subs.append(PtrSubCells(L, cart, r, q, sel, cq, csel, rest))
        origins.append(o)
    T = exch.LocalTransport(cart)
    for _ in range(3):
        exch.step(subs, T)
    assert 3 * 3 <= fake.launches <= 3 * 6      # one copy call per exchange that moves anything
    ref, cref = undivided_cells(pp, cells, rest, Lg, 3)
    Lg = np.array(Lg, float)
    got = np.full_like(ref, np.nan)
    cgot = np.full_like(cref, np.nan)
    for s, o in zip(subs, origins):
        got[s.ids] = np.concatenate([s.r + o, s.v], 1)
        cgot[s.cids] = np.concatenate([s.cr + o, s.cv], 2)
    d = got[:, :3] - ref[:, :3]
    d -= np.round(d / Lg) * Lg
    assert np.abs(d).max() < 1e-9 and np.abs(got[:, 3:] - ref[:, 3:]).max() < 1e-9
    d = cgot[..., :3] - cref[..., :3]
    d -= np.round(d / Lg) * Lg
    assert np.abs(d).max() < 1e-9 and np.abs(cgot[..., 3:] - cref[..., 3:]).max() < 1e-9


def test_subdomain_bag_addresses():
    """SubDomain.bag_ptrs: send bags one after another by the counts (kind 5:
    by the images received), receive bags at their fixed places (kind 5: by
    this rank's image counts), fixed bags for kind 2."""
    from ctc_b200 import exch

    class Fake:
        _ptrs = {0: (1000, [5000 + 64 * f for f in range(26)], [2] * 26, 32),
                 2: ([100 + f for f in range(26)], [200 + f for f in range(26)], [3] * 26, 4),
                 5: (7000, 9000, [8] * 26, 16)}
    counts = list(range(26))
    send, sent, recv, cap, unit = exch.SubDomain.bag_ptrs(Fake(), 0, counts)
    assert send[0] == 1000 and send[3] == 1000 + 32 * (0 + 1 + 2) and sent == counts
    assert recv[5] == 5000 + 64 * 5 and cap == [2] * 26 and unit == 32
    send, sent, recv, cap, unit = exch.SubDomain.bag_ptrs(Fake(), 2, None)
    assert send[4] == 104 and recv[4] == 204 and sent == [3] * 26 and unit == 4
    back = [2 * f for f in range(26)]
    send, sent, recv, cap, unit = exch.SubDomain.bag_ptrs(Fake(), 5, counts, back)
    assert sent == back and cap == counts and unit == 16
    assert send[2] == 7000 + 16 * (0 + 2) and recv[3] == 9000 + 16 * (0 + 1 + 2)
