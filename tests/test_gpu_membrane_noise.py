"""The membrane random force (rbc_force_set_rnd1 of src/rbc/force/imp/main.h,
src/rbc/force/dev/common.h:93-108) with counter-based normal numbers in place
of the reference's cuRAND ones: the sequence cannot match the reference's, so
these tests check what it must satisfy -- each edge's two directions take
equal and opposite forces (no momentum), the per-edge force has the variance
2 gammaC kBT / dt, a key gives the same forces every time and the next call
fresh ones."""
import numpy as np
import pytest

from ctc_b200 import systems

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

GC, KBT, DT = 10.0, 0.0444, 5e-4


def _noise_only(par):
    p = dict(par)
    for k in ("ks", "kb", "ka", "kd", "kv", "gammaT"):
        p[k] = 0.0
    p["gammaC"], p["kBT"] = GC, KBT
    return p


def _valence(tri, nv):
    deg = np.zeros(nv, np.int64)
    for c in range(3):
        np.add.at(deg, np.asarray(tri)[:, c], 1)
    return deg


def test_membrane_noise_statistics_and_momentum():
    import ctc_b200 as C
    L = (48, 48, 48)
    nc = 10
    pv, tri, par = systems.rbc_system(L, nc, seed=71)
    pv[:, 3:] = 0.0
    nv = len(pv) // nc
    mod = C.RbcForce(tri, nv, nc)
    mod.set_rnd(True, seed=7)
    pp = torch.as_tensor(pv, device="cuda")
    f1 = torch.zeros((len(pv), 3), device="cuda")
    mod.apply(C.RbcParams(**_noise_only(par)), pp, f1, dt=DT)
    f = f1.double().cpu().numpy()
    f0sq = float(np.float32(np.sqrt(np.float32(2.0 * GC * KBT / DT)))) ** 2
    # no momentum: every edge's two forces cancel, cell by cell
    per_cell = f.reshape(nc, nv, 3).sum(1)
    assert np.abs(per_cell).max() < 1e-6 * np.abs(f).sum() / nc
    # E|F_i|^2 = valence_i f0^2 (unit directions, unit-variance normals)
    deg = np.tile(_valence(tri, nv), nc)
    ratio = float(((f * f).sum(1) / deg).mean() / f0sq)
    assert abs(ratio - 1.0) < 0.05, ratio
    # the next call draws fresh numbers; a new module with the same seed repeats them
    f2 = torch.zeros_like(f1)
    mod.apply(C.RbcParams(**_noise_only(par)), pp, f2, dt=DT)
    assert not torch.equal(f1, f2)
    mod2 = C.RbcForce(tri, nv, nc)
    mod2.set_rnd(True, seed=7)
    f3 = torch.zeros_like(f1)
    mod2.apply(C.RbcParams(**_noise_only(par)), pp, f3, dt=DT)
    assert torch.equal(f1, f3)
    # off again: no force at all
    mod.set_rnd(False)
    f4 = torch.zeros_like(f1)
    mod.apply(C.RbcParams(**_noise_only(par)), pp, f4, dt=DT)
    assert f4.abs().max().item() == 0.0
    assert C.device_error() == 0


def test_sim_membrane_noise_momentum_and_graph_replay():
    """In the fast path (one key per step from the device trunk): the total
    momentum of solvent + membranes stays put, and graph replay gives the
    direct launches' result."""
    import ctc_b200 as C
    L = (16, 16, 16)
    ps = systems.solvent(L, seed=73)
    ps[:, 3:] -= ps[:, 3:].mean(0)
    pv, tri, par = systems.rbc_system(L, 1, seed=74)
    pv[:, 3:] = 0.0
    dpd = systems.dpd_params()
    out = []
    for graph in (False, True):
        sim = C.Sim(L, len(ps), C.DpdParams(*dpd), mass=1.0, dt=DT, rng=C.CTC_RNG_STABLE)
        sim.set_solvent(ps)
        sim.set_membranes(pv, tri, len(pv), par, C.DpdParams(0.0, 8.0, dpd[2], 0.25), mass=systems.RBC_MASS)
        sim.set_membrane_noise(True, seed=11)
        sim.set_graph(graph)
        sim.step(4)
        gs, gv = sim.get_solvent(), sim.get_membranes()
        p = gs[:, 3:].astype(np.float64).sum(0) + systems.RBC_MASS * gv[:, 3:].astype(np.float64).sum(0)
        p0 = ps[:, 3:].astype(np.float64).sum(0)
        assert np.abs(p - p0).max() < 1e-6 * np.abs(gs[:, 3:]).astype(np.float64).sum()
        out.append(gv)
        sim.close()
    assert np.abs(out[0] - out[1]).max() < 1e-4
    assert C.device_error() == 0
