"""Multi-process host logic of the decomposed solvent (no GPU): 2, 4 and 8
gloo ranks run the product's step orchestration (``exch.step``), cart
(``exch.Cart``) and transport (``exch.DistTransport``) over host tensors.
Each rank's subdomain is a numpy stand-in written here -- the same bins,
bags, shifts and record layout as the device kernels, with deterministic DPD
forces (no random term) in float64 -- and after three steps with migration
the ranks together hold exactly the undivided periodic box's state.  The
device kernels themselves are tested on the GPU (tests/test_gpu_exch.py)."""
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


def _rank_main(rank, world, port, dims, L, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import datetime

    import torch.distributed as dist
    from ctc_b200 import exch
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    cart = exch.Cart(dims)
    pp, Lg = _system(dims, L)
    c = np.floor((pp[:, :3] + np.array(Lg) / 2) / np.array(L)).astype(int)
    me = np.array(cart.coords(rank))
    sel = np.flatnonzero((c == me).all(1))
    o = -np.array(Lg) / 2 + (me + 0.5) * np.array(L)
    q = pp[sel].copy()
    q[:, :3] -= o
    sub = NumpySub(L, cart, rank, q, sel)
    T = exch.DistTransport(cart, rank)
    for _ in range(3):
        exch.step([sub], T)
    res = np.concatenate([sub.r + o, sub.v], 1)
    out.put((rank, sub.ids.tolist(), res.tolist()))
    dist.destroy_process_group()


def _system(dims, L):
    Lg = tuple(d * l for d, l in zip(dims, L))
    rng = np.random.default_rng(7)
    n = 3 * int(np.prod(Lg))
    r = -np.array(Lg) / 2 + rng.random((n, 3)) * np.array(Lg)
    v = rng.normal(0, 1.5, (n, 3))
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
    for rank, ids, st in res:
        got[ids] = np.array(st).reshape(-1, 6)
        seen[ids] += 1
    assert (seen == 1).all()
    d = got[:, :3] - ref[:, :3]
    d -= np.round(d / np.array(Lg)) * np.array(Lg)
    assert np.abs(d).max() < 1e-9
    assert np.abs(got[:, 3:] - ref[:, 3:]).max() < 1e-9
    # some particles changed rank on the way
    moved = sum(int((np.floor((np.array(st).reshape(-1, 6)[:, :3] + np.array(Lg) / 2) / np.array(L)) !=
                     np.floor((pp[ids, :3] + np.array(Lg) / 2) / np.array(L))).any(1).sum()) for _, ids, st in res)
    assert moved > 0


def test_cart_neighbours_are_symmetric():
    from ctc_b200 import exch
    for dims in [(1, 1, 1), (2, 1, 1), (3, 2, 1), (2, 2, 2), (4, 3, 2)]:
        cart = exch.Cart(dims)
        for r in range(cart.size):
            nb = cart.neighbours(r)
            assert cart.rank(cart.coords(r)) == r
            for f in range(26):
                assert cart.neighbours(nb[f])[exch.frag_anti(f)] == r
