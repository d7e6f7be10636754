"""Batched boxes: every box of a ctc_batch must be the system a single-box
ctc_sim of its size is -- same seeds, same box-local RNG keys, same wrap --
so a batch of boxes of uneven sizes (odd and even edges, some with a red
blood cell) is compared box by box with separate single-box runs."""
import numpy as np
import pytest

from ctc_b200 import systems

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

POS_TOL, VEL_TOL = 2e-6, 1e-3    # the system tests' per-step tolerances (force sums differ in order only)


def _boxes(seed=11):
    L = np.array([[8, 8, 8], [9, 9, 9], [12, 12, 12], [10, 10, 10], [7, 7, 7]], np.int32)
    rng = np.random.default_rng(seed)
    solv = [systems.solvent(tuple(l), seed=int(rng.integers(1 << 30))) for l in L]
    cells = np.array([1, 0, 1, 0, 0], np.int32)
    mem = {}
    for k in np.flatnonzero(cells):
        pv, tri, par = systems.rbc_system(tuple(L[k]), 1, seed=int(rng.integers(1 << 30)))
        mem[k] = pv
    return L, solv, cells, mem, tri, par


def _new_batch(L, solv, cells, mem, tri, par, dpd, fsi, bodyf):
    import ctc_b200 as C
    b = C.Batch(L, [len(p) for p in solv], C.DpdParams(*dpd), mass=1.0, dt=systems.DT, bodyf=bodyf)
    b.set_solvent(np.concatenate(solv))
    pv = np.concatenate([mem[k] for k in sorted(mem)])
    b.set_membranes(cells, pv, tri, 642, par, C.DpdParams(*fsi), mass=systems.RBC_MASS)
    return b


@pytest.mark.parametrize("graph", [False, True])
def test_batch_matches_single_boxes(graph):
    """Step by step: the batch against one single-box system per box, each
    single box restarted from the batch's state of the previous step (a
    particle within rounding of a cell face may change cell in one run and
    not in the other, which re-keys its pairs; restarting keeps the
    comparison to one step's arithmetic)."""
    import ctc_b200 as C
    L, solv, cells, mem, tri, par = _boxes()
    dpd = systems.dpd_params()
    fsi = (0.0, 8.0, dpd[2], 0.25)
    bodyf = (0.01, 0.0, 0.0)
    b = _new_batch(L, solv, cells, mem, tri, par, dpd, fsi, bodyf)
    b.set_graph(graph)
    sims = []
    for k in range(len(L)):
        s = C.Sim(tuple(L[k]), len(solv[k]), C.DpdParams(*dpd), mass=1.0, dt=systems.DT, bodyf=bodyf)
        sims.append(s)
    prev_s, prev_v = list(solv), dict(mem)
    for step in range(3):
        b.step(1)
        gs, gv = b.get_solvent(), b.get_membranes()
        o, ov = 0, 0
        for k, s in enumerate(sims):
            s.set_solvent(prev_s[k])
            if k in prev_v:
                s.set_membranes(prev_v[k], tri, 642, par, C.DpdParams(*fsi), mass=systems.RBC_MASS)
            s.step(1)
            rs = s.get_solvent()
            bs = gs[o:o + len(rs)]
            o += len(rs)
            assert np.abs(bs[:, :3] - rs[:, :3]).max() < POS_TOL, (step, k)
            assert np.abs(bs[:, 3:] - rs[:, 3:]).max() < VEL_TOL, (step, k)
            prev_s[k] = bs
            if k in prev_v:
                rv = s.get_membranes()
                bv = gv[ov:ov + len(rv)]
                ov += len(rv)
                assert np.abs(bv[:, :3] - rv[:, :3]).max() < POS_TOL, (step, k)
                assert np.abs(bv[:, 3:] - rv[:, 3:]).max() < VEL_TOL, (step, k)
                prev_v[k] = bv
        assert o == len(gs) and ov == len(gv)
    for s in sims:
        s.close()
    b.close()
    assert C.device_error() == 0


def test_batch_tune_leaves_state():
    """The autotuner times the pair kernels on the current state without
    advancing it or its generators."""
    import ctc_b200 as C
    L, solv, cells, mem, tri, par = _boxes(seed=12)
    dpd = systems.dpd_params()
    fsi = (0.0, 8.0, dpd[2], 0.25)
    out = []
    for tune in (False, True):
        b = _new_batch(L, solv, cells, mem, tri, par, dpd, fsi, (0, 0, 0))
        if tune:
            assert len(b.tune(reps=1)) == 4
        b.step(1)
        out.append((b.get_solvent(), b.get_membranes()))
        b.close()
    for x, y in zip(*out):
        assert np.abs(x[:, :3] - y[:, :3]).max() < POS_TOL
        assert np.abs(x[:, 3:] - y[:, 3:]).max() < VEL_TOL
    assert C.device_error() == 0


def test_batch_launch_shapes_agree():
    """Every launch shape the autotuner may pick computes the same forces."""
    import ctc_b200 as C
    L, solv, cells, mem, tri, par = _boxes(seed=13)
    dpd = systems.dpd_params()
    ref = None
    for shape in [(256, 4, 128, 2), (128, 2, 64, 4), (128, 8, 256, 2), (256, 8, 64, 4), (256, 2, 128, 4)]:
        b = C.Batch(L, [len(p) for p in solv], C.DpdParams(*dpd), dt=systems.DT)
        b.set_solvent(np.concatenate(solv))
        b.set_tune(shape)
        b.step(1)
        out = b.get_solvent()
        b.close()
        if ref is None:
            ref = out
        else:
            assert np.abs(out[:, :3] - ref[:, :3]).max() < POS_TOL
            assert np.abs(out[:, 3:] - ref[:, 3:]).max() < VEL_TOL
    assert C.device_error() == 0


@pytest.mark.parametrize("graph", [False, True])
def test_persistent_step_matches_launch_per_stage(graph):
    """The step as one persistent cooperative launch (grid-wide barriers
    between its stages, reference keys, membranes with FSI) against the same
    step as one launch per stage, three steps; with graph=True the step is
    one graph of that one launch."""
    import ctc_b200 as C
    L, solv, cells, mem, tri, par = _boxes(seed=14)
    dpd = systems.dpd_params()
    fsi = (0.0, 8.0, dpd[2], 0.25)
    bodyf = (0.01, 0.0, 0.0)
    out = []
    for persistent in (False, True):
        b = _new_batch(L, solv, cells, mem, tri, par, dpd, fsi, bodyf)
        b.set_persistent(persistent)
        b.set_graph(graph and persistent)
        for _ in range(3):
            b.step(1)
            out.append((persistent, b.get_solvent(), b.get_membranes()))
        if persistent:
            assert b.persistent_grid() >= 148
        b.close()
    assert C.device_error() == 0
    for k in range(3):
        (_, s0, v0), (_, s1, v1) = out[k], out[3 + k]
        assert np.abs(s0[:, :3] - s1[:, :3]).max() < POS_TOL * (k + 1)
        assert np.abs(s0[:, 3:] - s1[:, 3:]).max() < VEL_TOL
        assert np.abs(v0[:, :3] - v1[:, :3]).max() < POS_TOL * (k + 1)
        assert np.abs(v0[:, 3:] - v1[:, 3:]).max() < VEL_TOL


@pytest.mark.parametrize("build", [2, 3, 4])
def test_persistent_builds_match_launch_per_stage(build):
    """Each build of the persistent kernel (2, 3 or 4 blocks per SM: 128, 80
    or 64 registers) steps as the launch per stage does."""
    import ctc_b200 as C
    L, solv, cells, mem, tri, par = _boxes(seed=17)
    dpd = systems.dpd_params()
    fsi = (0.0, 8.0, dpd[2], 0.25)
    out = []
    for persistent in (0, build):
        b = _new_batch(L, solv, cells, mem, tri, par, dpd, fsi, (0.01, 0.0, 0.0))
        b.set_persistent(persistent)
        b.step(2)
        out.append((b.get_solvent(), b.get_membranes()))
        if persistent:
            assert b.persistent_grid() >= 148 * min(build, 2)
        b.close()
    (s0, v0), (s1, v1) = out
    assert np.abs(s0[:, :3] - s1[:, :3]).max() < 2 * POS_TOL
    assert np.abs(s0[:, 3:] - s1[:, 3:]).max() < VEL_TOL
    assert np.abs(v0[:, :3] - v1[:, :3]).max() < 2 * POS_TOL
    assert np.abs(v0[:, 3:] - v1[:, 3:]).max() < VEL_TOL
    assert C.device_error() == 0


def test_persistent_step_stable_keys():
    """The same with the stable keys (a second instantiation of the kernel)."""
    import ctc_b200 as C
    L, solv, cells, mem, tri, par = _boxes(seed=15)
    dpd = systems.dpd_params()
    out = []
    for persistent in (False, True):
        b = C.Batch(L, [len(p) for p in solv], C.DpdParams(*dpd), dt=systems.DT, rng=C.CTC_RNG_STABLE)
        b.set_solvent(np.concatenate(solv))
        b.set_persistent(persistent)
        b.step(2)
        out.append(b.get_solvent())
        b.close()
    assert np.abs(out[0][:, :3] - out[1][:, :3]).max() < 2 * POS_TOL
    assert np.abs(out[0][:, 3:] - out[1][:, 3:]).max() < VEL_TOL
    assert C.device_error() == 0


def test_persistent_barrier_wait_gives_up():
    """A block that never arrives at a grid barrier (a flag nothing sets)
    must not hang the device: the other blocks give up after their bounded
    wait, the step ends with CTC_DEV_WAIT_TIMEOUT in the device error word,
    and the context stays usable -- a fresh batch steps normally after it."""
    import ctc_b200 as C
    L, solv, cells, mem, tri, par = _boxes(seed=16)
    dpd = systems.dpd_params()
    fsi = (0.0, 8.0, dpd[2], 0.25)
    b = _new_batch(L, solv, cells, mem, tri, par, dpd, fsi, (0, 0, 0))
    b.set_persistent(True)
    b.step(1)
    assert C.device_error() == 0
    blocks = b.persistent_check(5)
    torch.cuda.synchronize()
    assert blocks >= 148
    assert C.device_error() == 5          # CTC_DEV_WAIT_TIMEOUT
    b.close()
    b = _new_batch(L, solv, cells, mem, tri, par, dpd, fsi, (0, 0, 0))
    b.set_persistent(True)
    b.step(2)
    torch.cuda.synchronize()
    assert C.device_error() == 0
    b.close()


def test_fused_count_bookkeeping_across_modes():
    """The update counts the next step's cells; every way of stepping keeps
    that right: direct steps, graph replays, a tuner call (which recounts), a
    persistent step (which counts itself) and back.  Without pair forces the
    motion is exact arithmetic (the membranes' internal forces are summed
    per vertex in a fixed order), so the states equal a run of direct steps
    bit for bit while particles and cells cross the boxes' faces."""
    import ctc_b200 as C
    L, solv, cells, mem, tri, par = _boxes(seed=19)
    rng = np.random.default_rng(20)
    solv = [p.copy() for p in solv]
    for p in solv:
        p[:, 3:] = rng.normal(0.0, 3.0, (len(p), 3)).astype(np.float32)
    zero = (0.0, 0.0, 0.0, 0.25)
    out = []
    for mixed in (False, True):
        b = _new_batch(L, solv, cells, mem, tri, par, zero, zero, (0.5, 0.0, 0.0))
        b.set_tune((128, 4, 128, 2))
        if not mixed:
            b.step(9)
        else:
            b.step(2)
            b.set_graph(True)
            b.step(2)
            b.tune(reps=1)
            b.set_tune((128, 4, 128, 2))
            b.step(2)
            b.set_persistent(True)
            b.step(1)
            b.set_persistent(False)
            b.step(2)
        out.append((b.get_solvent(), b.get_membranes()))
        b.close()
    (s0, v0), (s1, v1) = out
    assert np.array_equal(s0, s1)
    assert np.array_equal(v0, v1)
    assert C.device_error() == 0
