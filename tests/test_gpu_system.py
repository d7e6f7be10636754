"""The fused system step with membranes (solvent + red blood cells) against
the oracle's composition of the reference's modules, one step at a time."""
import numpy as np
import pytest

import oracle
from ctc_b200 import systems

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("bodyf", [None, (0.01, 0.0, 0.0)])
def test_rbc_system_steps_vs_oracle(bodyf):
    import ctc_b200 as C
    L = (16, 16, 16)
    ps = systems.solvent(L, seed=81)
    pv, tri, par = systems.rbc_system(L, 2, seed=82)
    nv = len(pv) // 2
    pv[:nv, 0] += L[0] / 2 - pv[:nv, 0].max() + 1.0        # one cell across the +x face
    dpd = systems.dpd_params()
    fsi = (0.0, 8.0, dpd[2], 0.25)
    sim = C.Sim(L, len(ps), C.DpdParams(*dpd), mass=1.0, dt=systems.DT, bodyf=bodyf or (0, 0, 0))
    sim.set_solvent(ps)
    sim.set_membranes(pv, tri, nv, par, C.DpdParams(*fsi), mass=systems.RBC_MASS)
    k0 = oracle.Kiss(0, 0, 0, 0)
    kh = [oracle.Kiss.halo(f) for f in range(26)]
    kf = oracle.Kiss(1908, 1409, 290, 12968)
    rs, rv = ps, pv
    for step in range(2):
        seeds = np.array([k0.get()] + [k.get() for k in kh], np.float32)
        assert np.array_equal(sim.next_seeds(), seeds)
        fseeds = (kf.get(), kf.get())
        sim.step(1)
        rs, rv = oracle.rbc_step(L, rs, rv, tri, nv, dpd, fsi, par, seeds, fseeds, bodyf, systems.DT, 1.0,
                                 systems.RBC_MASS)
        gs, gv = sim.get_solvent(), sim.get_membranes()
        assert gs.shape == rs.shape
        assert np.abs(gs[:, :3] - rs[:, :3]).max() < 2e-6
        assert np.abs(gs[:, 3:] - rs[:, 3:]).max() < 1e-3
        assert np.abs(gv[:, :3] - rv[:, :3]).max() < 2e-6
        assert np.abs(gv[:, 3:] - rv[:, 3:]).max() < 1e-3
        rs, rv = gs, gv          # continue from the device state (chaotic divergence)
    assert C.device_error() == 0


@pytest.mark.parametrize("edge", [12, 32])
def test_sim_graph_replay_matches_direct_launches(edge):
    """The step replayed as CUDA graphs gives the direct launches' result and
    advances the host mirrors of the trunks alike (membranes and contact on).
    In the 32^3 box (327,680 particles) both run the halo and solvent-membrane
    pairs on the second stream beside the bulk pairs; a third run, profiled,
    runs them one after the other, and all three agree."""
    import ctc_b200 as C
    L = (edge, edge, edge)
    ps = systems.solvent(L, seed=91)
    pv, tri, par = systems.rbc_system(L, 1, seed=92)
    dpd = systems.dpd_params()
    fsi = C.DpdParams(0.0, 8.0, dpd[2], 0.25)
    cnt = C.DpdLjParams(2.6666667, 8.0, dpd[2], 0.25, 0.3, 0.44)
    out = []
    for graph, prof in ((False, False), (True, False), (False, True)):
        sim = C.Sim(L, len(ps), C.DpdParams(*dpd), mass=1.0, dt=systems.DT, bodyf=(0.01, 0.0, 0.0))
        sim.set_solvent(ps)
        sim.set_membranes(pv, tri, len(pv), par, fsi, mass=systems.RBC_MASS)
        sim.set_contact(cnt)
        sim.set_graph(graph)
        sim.profile(prof)
        sim.step(4)
        sim.profile(False)
        seeds = sim.next_seeds()
        out.append((sim.get_solvent(), sim.get_membranes(), seeds))
        sim.close()
    (s0, v0, k0) = out[2]
    for s1, v1, k1 in out[:2]:
        assert np.array_equal(k0, k1)
        assert s0.shape == s1.shape
        assert np.abs(s0 - s1).max() < 1e-4 and np.abs(v0 - v1).max() < 1e-4
    assert C.device_error() == 0


def test_sim_tune_leaves_state():
    """The autotuner times the pair kernels on the current state without
    advancing it: the next steps match an untuned run's."""
    import ctc_b200 as C
    L = (12, 12, 12)
    ps = systems.solvent(L, seed=93)
    out = []
    for tune in (False, True):
        sim = C.Sim(L, len(ps), C.DpdParams(*systems.dpd_params()), mass=1.0, dt=systems.DT)
        sim.set_solvent(ps)
        sim.step(1)
        if tune:
            shape = sim.tune(reps=1)
            assert len(shape) == 5 and shape[0] in (128, 256) and shape[1] in (2, 4, 8) and shape[4] in (0, 1, 2)
            assert shape[2] in (64, 128, 256) and shape[3] in (2, 4)
        seeds = sim.next_seeds()
        sim.step(2)
        out.append((sim.get_solvent(), seeds))
        sim.close()
    assert np.array_equal(out[0][1], out[1][1])
    assert np.abs(out[0][0] - out[1][0]).max() < 1e-4
    assert C.device_error() == 0


def _rel_err(f, ref):
    f = np.asarray(f, np.float64).reshape(-1, 3)
    ref = np.asarray(ref, np.float64).reshape(-1, 3)
    mag = np.abs(ref).max(1)
    act = mag[mag > 0]
    floor = 0.1 * act.mean() if len(act) else 1.0
    return float((np.abs(f - ref).max(1) / np.maximum(mag, floor)).max())


@pytest.mark.parametrize("edge", [16, 32])
@pytest.mark.parametrize("case", ["membranes", "contact", "walls"])
def test_fused_step_forces_vs_modules(case, edge):
    """The force arrays of one fused step -- the solvent's (bulk + halo pairs,
    wall forces, FSI reactions) and the vertices' (wall forces and repulsion,
    FSI, contact, internal membrane forces on top) -- against the module entry
    points composed in the reference's order on the same state and seeds
    (each module held to the reference's own kernels at 1e-5): within 1e-5
    relative, max-norm per particle, so that no force term of the fused step
    can be dropped or doubled unseen.  The 32^3 box (327,680 particles) is
    large enough for the step to run the halo and solvent-membrane pairs on
    its second stream beside the bulk pairs; the 16^3 box runs them after."""
    import os

    import ctc_b200 as C
    from .test_gpu_wall import SDF
    L = (edge, edge, edge)
    dpd = systems.dpd_params()
    fsi = C.DpdParams(0.0, 8.0, dpd[2], 0.25)
    cnt = C.DpdLjParams(2.6666667, 8.0, dpd[2], 0.25, 0.3, 0.44)
    ps0 = systems.solvent(L, seed=101)
    pv, tri, par = systems.rbc_system(L, 2, seed=102)
    nv = len(pv) // 2
    sim = C.Sim(L, len(ps0), C.DpdParams(*dpd), mass=1.0, dt=systems.DT)
    sim.set_solvent(ps0)
    lam = 3.0
    if case == "walls":
        from ctc_b200 import mesh
        sdf = C.Sdf(L, path=os.path.join(SDF, "wall.dat"))
        wall = C.Wall(sdf, ps0)                           # the same freezing as the step's
        ps = wall.bulk
        sim.set_walls(sdf, C.wvel("cste"), lam=lam)
        assert np.array_equal(sim.get_solvent(), ps)
        X, F = mesh.rbc_template()                        # one cell in the channel, near a plate
        pv = np.zeros((len(X), 6), np.float32)
        pv[:, :3] = X
        pv[:, 2] += 4.2 * edge / 16                      # the plates scale with the box
        pv[:, 3:] = np.random.default_rng(103).normal(0, 0.3, (len(X), 3))
        tri, nv = F, len(X)
        A, V = mesh.area_volume(X, F)
        par = systems.rbc_params(A, V)
    else:
        ps = ps0
        pv[:nv, 0] += L[0] / 2 - pv[:nv, 0].max() + 1.0  # one cell across the +x face
        pv = oracle.rbc_wrap(L, pv, nv)                   # as the step's objects_distribute leaves it
    sim.set_membranes(pv, tri, nv, par, fsi, mass=systems.RBC_MASS)
    if case == "contact":
        pv[nv:, 2] = pv[:nv, 2] + 0.5                     # the second cell on top of the first
        pv[nv:, :2] = pv[:nv, :2]
        pv = oracle.rbc_wrap(L, pv, nv)
        sim.set_membranes(pv, tri, nv, par, fsi, mass=systems.RBC_MASS)
        sim.set_contact(cnt)
    seeds = sim.next_seeds()
    kf = oracle.Kiss(1908, 1409, 290, 12968)
    kc = oracle.Kiss(7119, 187, 18278, 15674)
    kw = oracle.Kiss(42, 42, 42, 42)
    sim.step(1)
    fs_step, fv_step = sim.forces()
    # the module entry points on the step's input state
    out, starts, counts, ids = C.Clist(L, len(ps)).build(torch.as_tensor(ps, device="cuda"))
    fs = torch.zeros((len(ps), 3), device="cuda")
    fv = torch.zeros((len(pv), 3), device="cuda")
    P = torch.as_tensor(pv, device="cuda")
    C.FluForces(L, len(ps)).apply_seeded(C.DpdParams(*dpd), out, starts, counts, seeds, fs, which=3)
    if case == "walls":
        wall.force(C.DpdParams(*dpd), out, fs, seed=kw.get())
        wall.force(fsi, P, fv, seed=kw.get())
        wall.repulse(lam, P, fv)
    C.Fsi(L, len(pv), len(ps)).apply_seeded(fsi, P, out, starts, counts, kf.get(), kf.get(), fv, fs)
    if case == "contact":
        C.Contact(L, len(pv)).apply_seeded(cnt, P, kc.get(), kc.get(), fv)
    C.RbcForce(tri, nv, len(pv) // nv).apply(C.RbcParams(**par), P, fv)
    torch.cuda.synchronize()
    assert C.device_error() == 0
    assert fv.abs().max().item() > 1.0 and fs.abs().max().item() > 1.0
    assert _rel_err(fs_step.cpu().numpy(), fs.cpu().numpy()) < 1e-5
    assert _rel_err(fv_step.cpu().numpy(), fv.cpu().numpy()) < 1e-5
    sim.close()


def test_fused_count_builds_the_same_cell_lists():
    """The update that counts the next step's cells (the default) against the
    cell-list build counting them itself.  Without pair forces the motion is
    exact arithmetic, so the states agree bit for bit while particles cross
    cells and periodic faces each step (direct steps, then graph replays, a
    tuner call in between that recounts); with forces they agree to the
    float atomics' order."""
    import ctc_b200 as C
    L = (16, 12, 8)
    ps = systems.solvent(L, seed=95)
    ps[:, 3:] = np.random.default_rng(96).normal(0.0, 3.0, (len(ps), 3)).astype(np.float32)
    for forces in (False, True):
        dpd = C.DpdParams(*systems.dpd_params()) if forces else C.DpdParams(0.0, 0.0, 0.0, 0.25)
        out = []
        for fused in (True, False):
            sim = C.Sim(L, len(ps), dpd, mass=1.0, dt=0.01, bodyf=(0.5, -0.25, 0.0))
            sim.set_fused_count(fused)
            sim.set_solvent(ps)
            sim.step(2)
            sim.set_graph(True)
            sim.step(3)
            sim.set_tune((128, 4, 128, 2))
            if fused:
                sim.tune(reps=1)
                sim.set_tune((128, 4, 128, 2))
            sim.step(3)
            out.append(sim.get_solvent())
            sim.close()
        a, b = out
        assert a.shape == b.shape == ps.shape
        if forces:
            assert np.abs(a - b).max() < 1e-3
        else:
            assert np.array_equal(a, b)
    assert C.device_error() == 0
