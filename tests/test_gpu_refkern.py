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
