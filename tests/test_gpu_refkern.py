"""GPU parity against the reference's own device code built from its sources
(oracle/_ref/librefkern.so via oracle/ref.mk): the pair RNG and the DPD pair
force.  This is what decides which FMA contraction of the RNG key sum the
reference executes, and it pins the product's pair arithmetic bit for bit."""
import numpy as np
import pytest

import oracle
from oracle import refkern
from ctc_b200 import systems

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refkern.available(), reason="oracle/_ref/librefkern.so not built")]


def dev(x):
    return torch.as_tensor(np.ascontiguousarray(x), device="cuda")


@pytest.mark.parametrize("unsigned", [False, True])
def test_rng_reference_kernel(unsigned):
    import ctc_b200 as C
    rng = np.random.default_rng(3)
    n = 300000
    u = rng.integers(0, 1 << 25, n).astype(np.int32)
    v = rng.integers(0, 1 << 25, n).astype(np.int32)
    k = oracle.Kiss(0, 0, 0, 0)
    for _ in range(3):
        seed = k.get()
        ref = refkern.rnd(seed, dev(u), dev(v), unsigned).cpu().numpy()
        ours = C.rnd_mean0var1(seed, dev(u), dev(v), unsigned=unsigned).cpu().numpy()
        orc = oracle.mean0var1_batch(seed, u, v, unsigned=unsigned)
        assert np.array_equal(ours.view(np.uint32), ref.view(np.uint32))
        assert np.array_equal(orc.view(np.uint32), ref.view(np.uint32))


def test_pair_force_reference_kernel():
    import ctc_b200 as C
    rng = np.random.default_rng(4)
    n = 200000
    d = rng.normal(size=(n, 3))
    d *= (rng.random(n) ** (1 / 3) / np.linalg.norm(d, axis=1))[:, None]   # inside the unit ball
    d[:100] *= 1e-4                                                           # r^2 < 1e-6 branch
    pa = rng.uniform(-8, 8, (n, 6)).astype(np.float32)
    pa[:, 3:] = rng.normal(0, 0.2, (n, 3))
    pb = pa.copy()
    pb[:, :3] = (pa[:, :3] - d).astype(np.float32)
    pb[:, 3:] = rng.normal(0, 0.2, (n, 3))
    r = rng.normal(0, 1, n).astype(np.float32)
    dpd = systems.dpd_params()
    ref = refkern.pair(dpd, dev(pa), dev(pb), dev(r)).cpu().numpy()
    ours = C.pair_force(C.DpdParams(*dpd), dev(pa), dev(pb), dev(r)).cpu().numpy()
    assert np.array_equal(ours.view(np.uint32), ref.view(np.uint32))


def _sorted(L, seed):
    pp = systems.solvent(L, seed=seed)
    counts, starts, order, ps = oracle.clist_build(L, pp)
    return ps, starts, counts


def _errs(f, ref):
    f = np.asarray(f, np.float64)
    ref = np.asarray(ref, np.float64)
    mag = np.abs(ref).max(1)
    return np.abs(f - ref).max(1) / np.maximum(mag, 0.1 * mag.mean())


@pytest.mark.parametrize("L", [(8, 8, 8), (16, 12, 10), (6, 6, 6)])
@pytest.mark.parametrize("which", [1, 2, 3])
def test_dpd_forces_reference_kernels(L, which):
    """bulk and halo forces against the reference's kernels on the same sorted
    particles and seeds: max-norm error per particle below 1e-5 relative"""
    import ctc_b200 as C
    ps, starts, counts = _sorted(L, 11)
    dpd = systems.dpd_params()
    seeds = np.random.default_rng(12).random(27).astype(np.float32)
    P, S, N = dev(ps), dev(starts), dev(counts)
    ref = torch.zeros((len(ps), 3), device="cuda")
    if which & 1:
        refkern.bulk(dpd, L, P, S, seeds[0], ref)
    if which & 2:
        refkern.halo(dpd, L, P, starts, counts, seeds[1:], ref)
    ours = torch.zeros((len(ps), 3), device="cuda")
    C.FluForces(L, len(ps)).apply_seeded(C.DpdParams(*dpd), P, S, N, seeds, ours, which=which)
    e = _errs(ours.cpu().numpy(), ref.cpu().numpy())
    assert e.max() < 1e-5, (e.max(), np.quantile(e, 0.999))


def test_bulk_kernel_faster_than_reference_kernel():
    """Speed bar: the bulk pair forces of a 64^3 box (2.6 M particles) on the
    same sorted particles, against the reference's own bulk kernel built for
    sm_100a (median of 5 timed launches each, CUDA events)."""
    import ctc_b200 as C
    L = (64, 64, 64)
    ps, starts, counts = _sorted(L, 13)
    dpd = systems.dpd_params()
    seeds = np.random.default_rng(14).random(27).astype(np.float32)
    P, S, N = dev(ps), dev(starts), dev(counts)
    out = torch.zeros((len(ps), 3), device="cuda")
    ff = C.FluForces(L, len(ps))

    def timed(fn):
        ts = []
        for _ in range(6):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(b))
        return float(np.median(ts[1:]))

    t_ref = timed(lambda: refkern.bulk(dpd, L, P, S, seeds[0], out))
    t_ours = timed(lambda: ff.apply_seeded(C.DpdParams(*dpd), P, S, N, seeds, out, which=1))
    print("bulk 64^3: reference kernel %.3f ms, this build %.3f ms" % (t_ref, t_ours))
    assert t_ours < t_ref, (t_ours, t_ref)


def _frag_lists(L, ps, starts, counts):
    """The exchanged fragments of a periodic box with itself as neighbour:
    fragment fid's local boundary particles (packed, with their sorted
    indices) and, as its remote fragment, the anti-fragment's packed particles
    and fragment-cell starts."""
    fr = refkern.fragments(L, starts, counts)
    P = dev(ps)
    lpp, lii, rpp, rst = [], [], [], []
    for fid in range(26):
        ii, _ = fr[fid]
        ia, ss = fr[oracle.frag_anti(fid)]
        lpp.append(P[torch.as_tensor(ii.astype(np.int64), device="cuda")].contiguous())
        lii.append(dev(ii))
        rpp.append(P[torch.as_tensor(ia.astype(np.int64), device="cuda")].contiguous())
        rst.append(dev(ss))
    return lpp, lii, rpp, rst


@pytest.mark.parametrize("L", [(8, 8, 8), (16, 12, 10), (6, 6, 6)])
def test_halo_from_exchanged_fragments_vs_reference_kernel(L):
    """fluforces_halo_prepare + _apply on the exchange's fragments
    (ctc_fluforces_halo_frags: the reference's LFrag26 / RFrag26 data) against
    the reference's own halo kernel on the same fragments and seeds, and
    against the module's halo from the cell lists: within 1e-5."""
    import ctc_b200 as C
    ps, starts, counts = _sorted(L, 21)
    dpd = systems.dpd_params()
    seeds = np.random.default_rng(22).random(27).astype(np.float32)
    lpp, lii, rpp, rst = _frag_lists(L, ps, starts, counts)
    ours = torch.zeros((len(ps), 3), device="cuda")
    C.FluForces(L, len(ps)).halo_frags(C.DpdParams(*dpd), lpp, lii, rpp, rst, ours, seeds26=seeds[1:])
    ref = torch.zeros((len(ps), 3), device="cuda")
    refkern.halo(dpd, L, dev(ps), starts, counts, seeds[1:], ref)
    e = _errs(ours.cpu().numpy(), ref.cpu().numpy())
    assert e.max() < 1e-5, e.max()
    mod = torch.zeros((len(ps), 3), device="cuda")
    C.FluForces(L, len(ps)).apply_seeded(C.DpdParams(*dpd), dev(ps), dev(starts), dev(counts), seeds, mod, which=2)
    assert _errs(ours.cpu().numpy(), mod.cpu().numpy()).max() < 1e-5
    assert C.device_error() == 0


def test_halo_from_fragments_draws_the_reference_trunks():
    """Without explicit seeds the 26 fragment seeds come from the module's
    trunks (src/fluforces/imp/ini.h:22-59), one draw each per call."""
    import ctc_b200 as C
    L = (8, 8, 8)
    ps, starts, counts = _sorted(L, 23)
    dpd = systems.dpd_params()
    lpp, lii, rpp, rst = _frag_lists(L, ps, starts, counts)
    mod = C.FluForces(L, len(ps))
    kh = [oracle.Kiss.halo(f) for f in range(26)]
    for _ in range(2):
        seeds = np.array([k.get() for k in kh], np.float32)
        ours = torch.zeros((len(ps), 3), device="cuda")
        mod.halo_frags(C.DpdParams(*dpd), lpp, lii, rpp, rst, ours)
        ref = torch.zeros((len(ps), 3), device="cuda")
        mod2 = C.FluForces(L, len(ps))
        mod2.halo_frags(C.DpdParams(*dpd), lpp, lii, rpp, rst, ref, seeds26=seeds)
        # particles of edge and corner cells take one atomic add per fragment
        assert _errs(ours.cpu().numpy(), ref.cpu().numpy()).max() < 1e-6
