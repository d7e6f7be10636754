"""GPU tests of the decomposed solvent (ctc_sub_*, ctc_b200/exch.py): the
ranks of a periodic cart run as emulated ranks on one device, their bags
moved by device copies (LocalTransport) -- the same pack, unpack and force
kernels a multi-GPU run uses, with NCCL only in place of the copies.

- one rank alone (all neighbours itself): its step's forces equal the
  periodic box's module entry points (held to the reference's kernels) at
  1e-5, reference keys;
- several ranks, reference keys: each rank's forces equal the module entry
  points fed the same exchanged fragments (fluforces_bulk_apply +
  fluforces_halo_apply on LFrag26 / RFrag26) with the rank's seeds and masks;
- several ranks, stable keys (the pair noise keyed by the particles' global
  ids): the forces equal the undivided box's at 1e-5 on positions on a
  2^-12 grid (every coordinate difference exact in both frames, so only the
  order of the sums differs), and a multi-step run with migration follows
  the undivided box's trajectory.
"""
import numpy as np
import pytest

from ctc_b200 import systems

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def mods():
    import ctc_b200 as C
    from ctc_b200 import exch
    return C, exch


def rel_err(f, ref):
    f = np.asarray(f, np.float64).reshape(-1, 3)
    ref = np.asarray(ref, np.float64).reshape(-1, 3)
    mag = np.abs(ref).max(1)
    return np.abs(f - ref).max(1) / np.maximum(mag, 0.1 * mag.mean())


def grid_solvent(Lg, seed, vstd=None, rho=10):
    """Particles of a [-Lg/2, Lg/2) box on a 2^-12 grid."""
    pp = systems.solvent(Lg, seed=seed, rho=rho)
    lo = systems.box_lo(np.asarray(Lg))
    q = np.floor((pp[:, :3] - lo) * 4096.0) / 4096.0 + lo
    pp[:, :3] = q.astype(np.float32)
    if vstd is not None:
        pp[:, 3:] = np.random.default_rng(seed + 1).normal(0, vstd, (len(pp), 3)).astype(np.float32)
    return pp


def split(pp, cart, L):
    """The particles of each rank in its subdomain's coordinates, and their
    global ids (index in pp)."""
    Lg = np.array(cart.dims) * np.array(L)
    lo = systems.box_lo(Lg)
    c = np.floor((pp[:, :3].astype(np.float64) - lo) / np.array(L)).astype(int)
    out = []
    for r in range(cart.size):
        cr = np.array(cart.coords(r))
        sel = np.flatnonzero((c == cr).all(1))
        o = lo + (cr + 0.5) * np.array(L)
        q = pp[sel].copy()
        q[:, :3] = (q[:, :3].astype(np.float64) - o).astype(np.float32)
        out.append((q, sel.astype(np.int32), o))
    return out


def sim_state(sim, n):
    """Cell-sorted state of a Sim with the ids of pos.w: (pp, ids, forces)."""
    import ctypes
    C, _ = mods()
    from ctc_b200 import _lib
    pos, vel, frc = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
    _lib.check(_lib.lib().ctc_sim_state(sim.h, ctypes.byref(pos), ctypes.byref(vel), ctypes.byref(frc), None))
    d = torch.device("cuda")
    p = C._wrap_dev(pos.value, 4 * n, torch.float32, d).reshape(n, 4).cpu().numpy()
    v = C._wrap_dev(vel.value, 4 * n, torch.float32, d).reshape(n, 4).cpu().numpy()
    f = C._wrap_dev(frc.value, 4 * n, torch.float32, d).reshape(n, 4).cpu().numpy()
    return np.concatenate([p[:, :3], v[:, :3]], 1), p[:, 3].copy().view(np.int32), f[:, :3]


def gather(subs, parts):
    """Every rank's state by global id: (pp in global coordinates, forces)."""
    n = sum(len(q) for q, _, _ in parts)
    pp = np.full((n, 6), np.nan, np.float64)
    ff = np.full((n, 3), np.nan, np.float64)
    seen = np.zeros(n, int)
    for s, (_, _, o) in zip(subs, parts):
        q, ids = s.get_solvent()
        f = s.forces()
        g = q.astype(np.float64)
        g[:, :3] += o
        pp[ids] = g
        ff[ids] = f
        seen[ids] += 1
    assert (seen == 1).all(), "every particle on exactly one rank"
    return pp, ff


@pytest.mark.parametrize("L", [(8, 8, 8), (12, 10, 8)])
def test_one_rank_forces_vs_modules(L):
    C, X = mods()
    cart = X.Cart((1, 1, 1))
    pp = systems.solvent(L, seed=5)
    n = len(pp)
    dpd = C.DpdParams(*systems.dpd_params())
    sub = X.SubDomain(L, cart, 0, n + 64, dpd, dt=0.0)
    sub.set_solvent(pp)
    seeds = sub.seeds()
    X.step([sub], X.LocalTransport(cart))
    torch.cuda.synchronize()
    ps, ids = sub.get_solvent()
    f = sub.forces()
    assert len(ps) == n and np.array_equal(np.sort(ids), np.arange(n))
    out, starts, counts, order = C.Clist(L, n).build(torch.as_tensor(ps, device="cuda"))
    assert np.array_equal(order.cpu().numpy(), np.arange(n))      # already cell-sorted, same order
    ff = torch.zeros((n, 3), device="cuda")
    C.FluForces(L, n).apply_seeded(dpd, out, starts, counts, seeds, ff, which=3)
    assert rel_err(f, ff.cpu().numpy()).max() < 1e-5
    assert C.device_error() == 0


def _phases_with_bags(subs, T):
    """One step of every rank (exch.step's phases), returning each rank's
    halo bags as the transport delivered them: (local records, their counts,
    received records, received counts, received fragment-cell starts)."""
    _, X = mods()
    R = X.SubDomain.REC
    for s in subs:
        s.distr_pack()
    counts = [s.distr_counts() for s in subs]
    rc = T.exchange_counts(counts)
    bags = [s.bags(0, c) for s, c in zip(subs, counts)]
    T.exchange([b[0] for b in bags], [b[1] for b in bags], rc, R).wait()
    for s, r in zip(subs, rc):
        s.distr_unpack(r)
    for s in subs:
        s.exch_pack()
    counts = [s.exch_counts() for s in subs]
    rc = T.exchange_counts(counts)
    bags = [s.bags(1, c) for s, c in zip(subs, counts)]
    fss = [s.bags(2, None) for s in subs]
    T.exchange([b[0] for b in bags], [b[1] for b in bags], rc, R).wait()
    T.exchange([b[0] for b in fss], [b[1] for b in fss], [b[2] for b in fss], 1).wait()
    snap = []
    for r, s in enumerate(subs):
        loc = [bags[r][0][f].clone().view(-1, 8) for f in range(26)]
        rem = [bags[r][1][j][:R * rc[r][j]].clone().view(-1, 8) for j in range(26)]
        rst = [fss[r][1][j].clone() for j in range(26)]
        snap.append((loc, counts[r], rem, rc[r], rst))
    for s in subs:
        s.bulk()
    for s, r in zip(subs, rc):
        s.halo_update(r)
    return snap


@pytest.mark.parametrize("dims", [(2, 1, 1), (2, 2, 1), (2, 2, 2)])
def test_ranks_reference_keys_vs_modules(dims):
    """Each rank's bulk + halo forces against fluforces_bulk_apply and
    fluforces_halo_apply on the fragments its neighbours sent, with the
    rank's seeds and key masks (src/fluforces/imp/ini.h:22-59)."""
    C, X = mods()
    L = (8, 8, 8)
    cart = X.Cart(dims)
    Lg = tuple(d * l for d, l in zip(dims, L))
    pp = systems.solvent(Lg, seed=11)
    parts = split(pp, cart, L)
    dpd = C.DpdParams(*systems.dpd_params())
    subs = [X.SubDomain(L, cart, r, len(pp), dpd, dt=0.0) for r in range(cart.size)]
    for s, (q, ids, _) in zip(subs, parts):
        s.set_solvent(q, ids)
    seeds = [s.seeds() for s in subs]
    snap = _phases_with_bags(subs, X.LocalTransport(cart))
    torch.cuda.synchronize()
    for r, s in enumerate(subs):
        ps, ids = s.get_solvent()
        n = len(ps)
        f = s.forces()
        where = {int(g): k for k, g in enumerate(ids)}
        loc, lc, rem, rc, rst = snap[r]
        aos = lambda t: t[:, [0, 1, 2, 4, 5, 6]].contiguous()
        lpp = [aos(loc[k]) for k in range(26)]
        lii = [torch.tensor([where[int(g)] for g in loc[k][:, 3].cpu().numpy().view(np.int32)], dtype=torch.int32,
                            device="cuda") for k in range(26)]
        rpp = [aos(rem[k]) for k in range(26)]
        out, starts, counts, order = C.Clist(L, n).build(torch.as_tensor(ps, device="cuda"))
        assert np.array_equal(order.cpu().numpy(), np.arange(n))
        mod = C.FluForces(L, n)
        mod.set_cart(cart.dims, cart.coords(r), r, cart.neighbours(r))
        ff = torch.zeros((n, 3), device="cuda")
        sd = np.zeros(27, np.float32)
        sd[0] = seeds[r][0]
        mod.apply_seeded(dpd, out, starts, counts, sd, ff, which=1)
        mod.halo_frags(dpd, lpp, lii, rpp, rst, ff, seeds26=seeds[r][1:])
        assert rel_err(f, ff.cpu().numpy()).max() < 1e-5, r
    assert C.device_error() == 0


@pytest.mark.parametrize("dims", [(2, 1, 1), (1, 2, 2), (2, 2, 2)])
def test_ranks_stable_keys_forces_equal_undivided_box(dims):
    C, X = mods()
    L = (8, 8, 8)
    cart = X.Cart(dims)
    Lg = tuple(d * l for d, l in zip(dims, L))
    pp = grid_solvent(Lg, seed=21)
    n = len(pp)
    dpd = C.DpdParams(*systems.dpd_params())
    sim = C.Sim(Lg, n, dpd, dt=0.0, rng=C.CTC_RNG_STABLE)
    sim.set_solvent(pp)
    sim.step(1)
    torch.cuda.synchronize()
    _, sids, sf = sim_state(sim, n)
    ref = np.empty((n, 3))
    ref[sids] = sf
    parts = split(pp, cart, L)
    subs = [X.SubDomain(L, cart, r, n, dpd, dt=0.0, rng=C.CTC_RNG_STABLE) for r in range(cart.size)]
    for s, (q, ids, _) in zip(subs, parts):
        s.set_solvent(q, ids)
    X.step(subs, X.LocalTransport(cart))
    torch.cuda.synchronize()
    _, ff = gather(subs, parts)
    assert rel_err(ff, ref).max() < 1e-5
    assert C.device_error() == 0


def test_ranks_steps_with_migration_follow_undivided_box():
    """Six steps of a 2 x 2 x 2 cart with fast particles (a few percent cross
    a face each step) and a body force, against the undivided box with the
    same stable keys: every particle on the rank whose subdomain holds it,
    positions within 1e-5 (99.9 %) and velocities within 1e-3 (99 %) of the
    undivided run.  The two frames round positions differently (subdomain
    against box coordinates) and a pair within rounding of the cutoff, where
    (1 - r)^0.25 has an unbounded slope, amplifies that into the few larger
    deviations the maxima allow."""
    C, X = mods()
    L = (8, 8, 8)
    dims = (2, 2, 2)
    cart = X.Cart(dims)
    Lg = tuple(d * l for d, l in zip(dims, L))
    pp = grid_solvent(Lg, seed=31, vstd=2.0)
    n = len(pp)
    dpd = C.DpdParams(*systems.dpd_params())
    dt, bodyf, K = 0.01, (0.5, 0.0, 0.0), 6
    sim = C.Sim(Lg, n, dpd, dt=dt, bodyf=bodyf, rng=C.CTC_RNG_STABLE)
    sim.set_solvent(pp)
    sim.step(K)
    torch.cuda.synchronize()
    sp, sids, _ = sim_state(sim, n)
    ref = np.empty((n, 6))
    ref[sids] = sp
    parts = split(pp, cart, L)
    subs = [X.SubDomain(L, cart, r, n, dpd, dt=dt, bodyf=bodyf, rng=C.CTC_RNG_STABLE, maxd=40.0)
            for r in range(cart.size)]
    for s, (q, ids, _) in zip(subs, parts):
        s.set_solvent(q, ids)
    T = X.LocalTransport(cart)
    moved = 0
    for k in range(K):
        before = [set(s.get_solvent()[1].tolist()) for s in subs]
        X.step(subs, T)
        torch.cuda.synchronize()
        moved += sum(len(b - set(s.get_solvent()[1].tolist())) for b, s in zip(before, subs))
    assert moved > 0.01 * n, moved
    got, _ = gather(subs, parts)
    # the undivided box's positions wrapped into [lo, lo + Lg)
    lo = systems.box_lo(np.asarray(Lg))
    dx = got[:, :3] - ref[:, :3]
    dx -= np.round(dx / np.array(Lg)) * np.array(Lg)
    dx = np.abs(dx).max(1)
    assert np.quantile(dx, 0.999) < 1e-5 and dx.max() < 2e-3, (np.quantile(dx, 0.999), dx.max())
    dv = np.abs(got[:, 3:] - ref[:, 3:]).max(1)
    assert np.quantile(dv, 0.99) < 1e-3 and dv.max() < 0.2, (np.quantile(dv, 0.99), dv.max())
    # each rank holds the particles its subdomain held before the last
    # update (they migrate at the start of the next step, as the reference's)
    for s in subs:
        q, _ = s.get_solvent()
        assert (np.abs(q[:, 3:]) * dt < 0.5).all()
        assert (q[:, :3] >= -4.5).all() and (q[:, :3] < 4.5).all()
    assert lo is not None and C.device_error() == 0


def test_bag_capacity_overflow_is_an_error():
    """A migration bag beyond its capacity (maxd too small for the flux) is
    reported as CTC_ERR_CAPACITY before any exchange: a quarter of the
    particles cross the +x face in one step, its bag holds maxd per face cell."""
    C, X = mods()
    from ctc_b200._lib import CtcError
    L = (8, 8, 8)
    cart = X.Cart((2, 1, 1))
    pp = systems.solvent(L, seed=3)
    pp[:, 3] += 200.0           # 2 cells per step along +x
    dpd = C.DpdParams(*systems.dpd_params())
    sub = X.SubDomain(L, cart, 0, len(pp), dpd, dt=0.01, maxd=12.0)
    sub.set_solvent(pp)
    sub.distr_pack()
    assert sub.distr_counts() == [0] * 26
    sub.distr_unpack([0] * 26)
    sub.exch_pack()
    sub.bulk()
    sub.exch_counts()
    sub.halo_update([0] * 26)
    sub.distr_pack()
    with pytest.raises(CtcError, match="capacity"):
        sub.distr_counts()
    assert C.device_error() == 0


def test_dist_transport_one_rank_nccl_equals_local():
    """The NCCL transport of a one-rank cart (every bag a message to itself,
    copied on the device) steps the subdomain as the in-process transport
    does."""
    import datetime
    import socket

    import torch.distributed as dist
    C, X = mods()
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    dist.init_process_group("nccl", init_method="tcp://127.0.0.1:%d" % port, rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        L = (8, 8, 8)
        cart = X.Cart((1, 1, 1))
        pp = systems.solvent(L, seed=41)
        dpd = C.DpdParams(*systems.dpd_params())
        out = []
        for T in (X.LocalTransport(cart), X.DistTransport(cart, 0, device=torch.device("cuda"))):
            sub = X.SubDomain(L, cart, 0, len(pp) + 64, dpd)
            sub.set_solvent(pp)
            for _ in range(3):
                X.step([sub], T)
            torch.cuda.synchronize()
            out.append(sub.get_solvent())
        # the same particles in the same order; the float atomics of the force
        # sums leave the last bits to the order in which the pairs land
        assert np.array_equal(out[0][1], out[1][1])
        assert np.abs(out[0][0][:, :3] - out[1][0][:, :3]).max() < 1e-6
        assert np.abs(out[0][0][:, 3:] - out[1][0][:, 3:]).max() < 1e-4
    finally:
        dist.destroy_process_group()
    assert C.device_error() == 0


# -- membranes in the decomposed step ------------------------------------------
def grid_cells(centres, seed, drift=(0.0, 0.0, 0.0)):
    """RBCs (642 vertices) around the given centres, randomly rotated, on the
    2^-12 grid: (pv (nc*642, 6), triangles, parameters)."""
    from ctc_b200 import mesh
    X, F = mesh.rbc_template(7.82)
    rng = np.random.default_rng(seed)
    r = np.concatenate([X @ mesh.random_rotation(rng).T + np.asarray(c) for c in centres])
    pv = np.zeros((len(r), 6), np.float32)
    pv[:, :3] = np.floor(r * 4096.0) / 4096.0
    pv[:, 3:] = rng.normal(0.0, np.sqrt(systems.KBT / systems.RBC_MASS), (len(r), 3)) + np.asarray(drift)
    A, V = mesh.area_volume(X, F)
    return pv, F, systems.rbc_params(A, V)


def split_cells(pv, nv, cart, L):
    """Every rank's cells (the rank whose subdomain holds the centre of the
    cell's bounding box) in its subdomain's coordinates, and their ids."""
    Lg = np.array(cart.dims) * np.array(L)
    lo = systems.box_lo(Lg)
    r = pv[:, :3].astype(np.float64).reshape(-1, nv, 3)
    c = 0.5 * (r.min(1) + r.max(1))
    b = np.floor((c - lo) / np.array(L)).astype(int)
    out = []
    for k in range(cart.size):
        ck = np.array(cart.coords(k))
        sel = np.flatnonzero((b == ck).all(1))
        o = lo + (ck + 0.5) * np.array(L)
        q = pv.reshape(-1, nv, 6)[sel].copy()
        q[:, :, :3] = (q[:, :, :3].astype(np.float64) - o).astype(np.float32)
        out.append((q.reshape(-1, 6), sel.astype(np.int32), o))
    return out


def sim_membranes(sim, nvt):
    """(positions, velocities, forces) of a Sim's vertices, cell after cell."""
    import ctypes
    C, _ = mods()
    from ctc_b200 import _lib
    p, v, f = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
    _lib.check(_lib.lib().ctc_sim_membrane_state(sim.h, ctypes.byref(p), ctypes.byref(v), ctypes.byref(f)))
    d = torch.device("cuda")
    get = lambda a: C._wrap_dev(a.value, 4 * nvt, torch.float32, d).reshape(nvt, 4)[:, :3].cpu().numpy()
    return get(p), get(v), get(f)


def _mem_setup(dims, L, centres, seed, dt, bodyf=(0.0, 0.0, 0.0), drift=(0.0, 0.0, 0.0), vstd=None):
    C, X = mods()
    cart = X.Cart(dims)
    Lg = tuple(d * l for d, l in zip(dims, L))
    pp = grid_solvent(Lg, seed=seed, vstd=vstd)
    pp[:, 3:] += np.asarray(drift, np.float32)      # the solvent flows with the cells
    pv, tri, par = grid_cells(centres, seed + 1, drift)
    nv = 642
    dpd = C.DpdParams(*systems.dpd_params())
    fsi = C.DpdParams(*systems.dpd_params())
    sim = C.Sim(Lg, len(pp), dpd, dt=dt, bodyf=bodyf, rng=C.CTC_RNG_STABLE)
    sim.set_solvent(pp)
    sim.set_membranes(pv, tri, nv, par, fsi, mass=systems.RBC_MASS)
    parts = split(pp, cart, L)
    cparts = split_cells(pv, nv, cart, L)
    subs = [X.SubDomain(L, cart, r, len(pp), dpd, dt=dt, bodyf=bodyf, rng=C.CTC_RNG_STABLE, maxd=40.0)
            for r in range(cart.size)]
    for s, (q, ids, _), (cq, cids, _) in zip(subs, parts, cparts):
        s.set_solvent(q, ids)
        s.set_membranes(cq, cids, tri, nv, par, fsi, maxc=len(centres), mass=systems.RBC_MASS)
    return cart, pp, pv, sim, subs, parts, cparts


def gather_membranes(subs, parts, nvt, nv):
    """Every rank's vertices by global vertex id: (pv in global coordinates,
    forces, the rank of each cell)."""
    pv = np.full((nvt, 6), np.nan)
    ff = np.full((nvt, 3), np.nan)
    owner = np.full(nvt // nv, -1)
    for r, (s, (_, _, o)) in enumerate(zip(subs, parts)):
        q, cids = s.get_membranes()
        f, vids = s.membrane_forces()
        assert np.array_equal(vids, (cids[:, None] * nv + np.arange(nv)).reshape(-1))
        g = q.astype(np.float64)
        g[:, :3] += o
        pv[vids] = g
        ff[vids] = f
        assert (owner[cids] == -1).all(), "every cell on exactly one rank"
        owner[cids] = r
    assert (owner >= 0).all()
    return pv, ff, owner


@pytest.mark.parametrize("dims,L,centres", [
    ((2, 1, 1), (16, 16, 16), [(0.3, 0.2, -0.4), (-15.7, 3.1, 2.2), (-8.0, -4.0, 4.5)]),
    ((2, 2, 1), (16, 16, 16), [(0.3, 0.4, -0.4), (-15.6, -15.7, 2.2), (8.2, -8.0, -6.3), (-7.9, 7.6, 5.1)]),
])
def test_ranks_membranes_forces_equal_undivided_box(dims, L, centres):
    """Cells straddling the faces between ranks (their vertices' images cross
    for FSI, the forces on the images come back): solvent and vertex forces
    equal the undivided box's at 1e-5 with stable keys, positions on the
    2^-12 grid."""
    C, X = mods()
    cart, pp, pv, sim, subs, parts, cparts = _mem_setup(dims, L, centres, 51, dt=0.0)
    n, nv, nvt = len(pp), 642, len(pv)
    sim.step(1)
    torch.cuda.synchronize()
    _, sids, sf = sim_state(sim, n)
    ref = np.empty((n, 3))
    ref[sids] = sf
    _, _, mref = sim_membranes(sim, nvt)
    X.step(subs, X.LocalTransport(cart))
    torch.cuda.synchronize()
    _, ff = gather(subs, parts)
    _, mf, owner = gather_membranes(subs, parts, nvt, nv)
    # the FSI reactions reach the solvent on the ranks across the faces
    assert rel_err(ff, ref).max() < 1e-5
    assert rel_err(mf, mref).max() < 1e-5
    assert len(set(owner.tolist())) > 1
    assert C.device_error() == 0


def test_ranks_membranes_migrate_and_follow_undivided_box():
    """Solvent and cells flowing along x (0.2 per step): a cell crosses the
    face between the two ranks, another the periodic face, and both change
    rank; six steps with a body force: every cell on the rank that holds its bounding-box centre, and the
    vertices and the solvent follow the undivided box's run."""
    C, X = mods()
    dims, L = (2, 1, 1), (16, 16, 16)
    centres = [(-0.45, 0.2, -0.4), (15.55, 3.1, 2.2), (-8.0, -4.0, 4.5)]
    dt, K = 0.01, 6
    cart, pp, pv, sim, subs, parts, cparts = _mem_setup(dims, L, centres, 61, dt=dt, bodyf=(0.5, 0.0, 0.0),
                                                        drift=(20.0, 0.0, 0.0), vstd=1.0)
    n, nv, nvt = len(pp), 642, len(pv)
    owners = []
    T = X.LocalTransport(cart)
    for k in range(K):
        X.step(subs, T)
        torch.cuda.synchronize()
        owners.append(gather_membranes(subs, parts, nvt, nv)[2])
    sim.step(K)
    torch.cuda.synchronize()
    assert owners[0][0] == 0 and owners[-1][0] == 1, owners
    assert owners[0][1] == 1 and owners[-1][1] == 0, owners
    mp, mv, _ = sim_membranes(sim, nvt)
    got, _, _ = gather_membranes(subs, parts, nvt, nv)
    Lg = np.array(cart.dims) * np.array(L)
    dx = got[:, :3] - mp
    dx -= np.round(dx / Lg) * Lg
    dx = np.abs(dx).max(1)
    assert np.quantile(dx, 0.999) < 1e-4 and dx.max() < 2e-3, (np.quantile(dx, 0.999), dx.max())
    dv = np.abs(got[:, 3:] - mv).max(1)
    assert np.quantile(dv, 0.99) < 1e-2 and dv.max() < 0.2, (np.quantile(dv, 0.99), dv.max())
    sp, sids, _ = sim_state(sim, n)
    ref = np.empty((n, 6))
    ref[sids] = sp
    sg, _ = gather(subs, parts)
    dx = sg[:, :3] - ref[:, :3]
    dx -= np.round(dx / Lg) * Lg
    dx = np.abs(dx).max(1)
    assert np.quantile(dx, 0.999) < 1e-4 and dx.max() < 2e-3, (np.quantile(dx, 0.999), dx.max())
    assert C.device_error() == 0


def test_rank_without_cells_takes_images_and_a_cell():
    """Every cell starts on rank 0 of a 2 x 1 x 1 cart: rank 1 holds none, yet
    evaluates FSI for the images that cross to it and sends their forces
    back (forces equal to the undivided box's at dt = 0); then, flowing along
    x, a cell migrates into the empty rank."""
    C, X = mods()
    dims, L = (2, 1, 1), (16, 16, 16)
    centres = [(-0.3, 0.2, -0.4), (-8.0, -4.0, 4.5)]
    cart, pp, pv, sim, subs, parts, cparts = _mem_setup(dims, L, centres, 71, dt=0.0)
    assert len(cparts[1][1]) == 0 and len(cparts[0][1]) == 2
    n, nv, nvt = len(pp), 642, len(pv)
    sim.step(1)
    torch.cuda.synchronize()
    _, sids, sf = sim_state(sim, n)
    ref = np.empty((n, 3))
    ref[sids] = sf
    _, _, mref = sim_membranes(sim, nvt)
    X.step(subs, X.LocalTransport(cart))
    torch.cuda.synchronize()
    _, ff = gather(subs, parts)
    _, mf, owner = gather_membranes(subs, parts, nvt, nv)
    assert (owner == 0).all()
    assert rel_err(ff, ref).max() < 1e-5
    assert rel_err(mf, mref).max() < 1e-5
    # the flow carries the first cell across x = 0 into rank 1
    cart, pp, pv, sim, subs, parts, cparts = _mem_setup(dims, L, centres, 71, dt=0.01, drift=(20.0, 0.0, 0.0),
                                                        vstd=1.0)
    T = X.LocalTransport(cart)
    for _ in range(4):
        X.step(subs, T)
    torch.cuda.synchronize()
    _, _, owner = gather_membranes(subs, parts, nvt, nv)
    assert owner[0] == 1 and owner[1] == 0, owner
    assert C.device_error() == 0


def test_membrane_bag_capacity_overflow_is_an_error():
    """More cells leaving through one face than a cell bag holds (a quarter
    of maxc, at least 4) is CTC_ERR_CAPACITY at the counts, before any
    exchange."""
    C, X = mods()
    from ctc_b200._lib import CtcError
    dims, L = (2, 1, 1), (24, 24, 24)
    # six cells just inside the +x face, moved beyond it
    centres = [(-0.2, y, z) for y in (-8.0, 0.0, 8.0) for z in (-6.0, 6.0)]
    Lg = (48, 24, 24)
    pv, tri, par = grid_cells(centres, 81)
    nv = 642
    cartX = X.Cart(dims)
    cp = split_cells(pv, nv, cartX, L)
    assert len(cp[0][1]) == 6
    pp = grid_solvent(Lg, seed=81)
    parts = split(pp, cartX, L)
    dpd = C.DpdParams(*systems.dpd_params())
    sub = X.SubDomain(L, cartX, 0, len(pp), dpd, dt=0.0)
    sub.set_solvent(parts[0][0], parts[0][1])
    q = cp[0][0].copy()
    q[:, 0] += 0.5                  # every centre now beyond the face
    sub.set_membranes(q, cp[0][1], tri, nv, par, C.DpdParams(*systems.dpd_params()), maxc=6,
                      mass=systems.RBC_MASS)
    sub.mem_distr_pack()
    with pytest.raises(CtcError, match="capacity"):
        sub.mem_distr_counts()
    assert C.device_error() == 0


def test_dist_transport_one_rank_nccl_with_cells_equals_local():
    """The NCCL transport of a one-rank cart with cells (they leave and
    re-enter through the periodic faces, their images come back to the rank
    itself) steps as the in-process transport does."""
    import datetime
    import socket

    import torch.distributed as dist
    C, X = mods()
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    dist.init_process_group("nccl", init_method="tcp://127.0.0.1:%d" % port, rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        L = (16, 16, 16)
        cart = X.Cart((1, 1, 1))
        pp = grid_solvent(L, seed=91, vstd=1.0)
        pp[:, 3] += 20.0
        pv, tri, par = grid_cells([(7.9, 0.1, 0.2), (-3.0, 4.0, -7.5)], 92, drift=(20.0, 0.0, 0.0))
        dpd = C.DpdParams(*systems.dpd_params())
        out = []
        for T in (X.LocalTransport(cart), X.DistTransport(cart, 0, device=torch.device("cuda"))):
            sub = X.SubDomain(L, cart, 0, len(pp) + 64, dpd, dt=0.01)
            sub.set_solvent(pp)
            sub.set_membranes(pv, np.arange(2, dtype=np.int32), tri, 642, par, C.DpdParams(*systems.dpd_params()),
                              maxc=4, mass=systems.RBC_MASS)
            for _ in range(4):
                X.step([sub], T)
            torch.cuda.synchronize()
            out.append((sub.get_solvent(), sub.get_membranes()))
        (s0, m0), (s1, m1) = out
        assert np.array_equal(s0[1], s1[1]) and np.array_equal(m0[1], m1[1])
        assert np.abs(s0[0][:, :3] - s1[0][:, :3]).max() < 1e-5
        assert np.abs(m0[0][:, :3] - m1[0][:, :3]).max() < 1e-5
        assert np.abs(m0[0][:, 3:] - m1[0][:, 3:]).max() < 1e-2
    finally:
        dist.destroy_process_group()
    assert C.device_error() == 0
