"""Juelicher bending (rbc_force_set_bending "juelicher",
src/rbc/force/bending/juelicher) on the device: against the oracle (both in
double, per-vertex gathers on the device, the reference's per-edge scatter in
the oracle) and against the reference's own kernels built from its sources
(oracle/_ref/librefkern.so), which keep the per-vertex area, length x angle,
angles and forces in float and add them with float atomics.

Tolerances (per-vertex max-norm error relative to the vertex's force, floored
at 0.1 x the mean): 1e-6 against the oracle (measured 5.8e-8, the float
output); 5e-5 against the reference's kernels, whose float intermediates and
unordered float sums carry errors of about 1e-7 of the per-edge terms that,
on a vertex, mostly cancel (measured 1.0e-5 and 1.9e-5 on the two templates,
the same against the oracle as against the device)."""
import os

import numpy as np
import pytest

import oracle
from oracle import refkern
from ctc_b200 import mesh, systems

from .conftest import GOLDEN

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def dev(x):
    return torch.as_tensor(np.ascontiguousarray(x), device="cuda")


def rel_err(f, ref):
    f = np.asarray(f, np.float64).reshape(-1, 3)
    ref = np.asarray(ref, np.float64).reshape(-1, 3)
    mag = np.abs(ref).max(1)
    return float((np.abs(f - ref).max(1) / np.maximum(mag, 0.1 * mag.mean())).max())


def _cells(nc, seed, template="642.off", noise=0.02):
    if template == "642.off":
        V, F = mesh.read_off(os.path.join(GOLDEN, "rbc.642.off"))
    else:
        V, F = mesh.rbc_template()
    rng = np.random.default_rng(seed)
    r = np.concatenate([V @ mesh.random_rotation(rng).T + rng.uniform(-5, 5, 3) for _ in range(nc)])
    r += rng.normal(0, noise, r.shape)
    pp = np.zeros((len(r), 6), np.float32)
    pp[:, :3] = r
    pp[:, 3:] = rng.normal(0, 0.3, (len(r), 3))
    A, Vol = mesh.area_volume(V, F)
    return pp, F, len(V), systems.rbc_params(A * 1.01, Vol * 0.99)


def _only_bending(par):
    p = dict(par)
    for k in ("ks", "kb", "ka", "kd", "kv", "gammaC", "gammaT", "kBT"):
        p[k] = 0.0
    return p


@pytest.mark.parametrize("template,noise", [("642.off", 0.02), ("evans-fung", 0.02), ("642.off", 0.1)])
def test_juelicher_vs_oracle(template, noise):
    import ctc_b200 as C
    pp, F, nv, par = _cells(3, 5, template, noise)
    ref = oracle.juelicher_forces(F, nv, pp)
    mod = C.RbcForce(F, nv, 4)
    mod.set_bending("juelicher")
    ff = torch.zeros((len(pp), 3), device="cuda")
    mod.apply(C.RbcParams(**_only_bending(par)), dev(pp), ff)
    assert C.device_error() == 0
    err = rel_err(ff.cpu().numpy(), ref)
    print("juelicher device vs oracle:", err)
    assert err < 1e-6


def _dev_juelicher(C, F, nv, pp, par):
    mod = C.RbcForce(F, nv, 4)
    mod.set_bending("juelicher")
    ff = torch.zeros((len(pp), 3), device="cuda")
    mod.apply(C.RbcParams(**_only_bending(par)), dev(pp), ff)
    return ff.cpu().numpy()


@pytest.mark.skipif(not refkern.available(), reason="oracle/_ref/librefkern.so not built")
@pytest.mark.parametrize("template", ["642.off", "evans-fung"])
def test_juelicher_vs_reference_kernels(template):
    """The reference's nine kernels sum their per-triangle and per-edge
    terms in float with atomics, in an order that changes from run to run;
    this build gathers per vertex in double.  Measured against the FP64
    oracle: this build 6e-8, the reference's kernels 1.2e-5 and 2.4e-5 (the
    two templates); two runs of the reference's kernels on the same input
    differ from each other by 1.4e-5 and 2.0e-5.  The gap between the two
    builds is the reference's own float accumulation, which varies from run
    to run by more than 1e-5: no build can reproduce it more closely, so the
    bar is 5e-5 here and this build is held to 1e-6 of the oracle."""
    import ctc_b200 as C
    pp, F, nv, par = _cells(4, 6, template)
    fr = torch.zeros((len(pp), 3), device="cuda")
    refkern.juelicher(F, nv, dev(pp), fr)
    ref = fr.cpu().numpy()
    fr2 = torch.zeros((len(pp), 3), device="cuda")
    refkern.juelicher(F, nv, dev(pp), fr2)
    e_runs = rel_err(fr2.cpu().numpy(), ref)
    orc = oracle.juelicher_forces(F, nv, pp)
    e_orc = rel_err(ref, orc)
    e_me = rel_err(_dev_juelicher(C, F, nv, pp, par), orc)
    print("juelicher reference kernels: run to run", e_runs, "vs FP64 oracle", e_orc, "; this build vs oracle", e_me)
    assert e_me < 1e-6 and e_me < e_orc
    mod = C.RbcForce(F, nv, 4)
    mod.set_bending("juelicher")
    ff = torch.zeros((len(pp), 3), device="cuda")
    mod.apply(C.RbcParams(**_only_bending(par)), dev(pp), ff)
    e_dev = rel_err(ff.cpu().numpy(), ref)
    print("juelicher reference kernels vs oracle:", e_orc, " device vs reference kernels:", e_dev)
    assert e_orc < 5e-5
    assert e_dev < 5e-5


def test_juelicher_with_the_other_membrane_forces():
    """The module adds the Juelicher bending to the spring, area, volume and
    viscous forces (Kantor's term off)."""
    import ctc_b200 as C
    pp, F, nv, par = _cells(2, 7)
    ref = oracle.rbc_forces(F, nv, pp, dict(par, kb=0.0), mode=0) + oracle.juelicher_forces(F, nv, pp)
    mod = C.RbcForce(F, nv, 2)
    mod.set_bending("juelicher")
    ff = torch.zeros((len(pp), 3), device="cuda")
    mod.apply(C.RbcParams(**par), dev(pp), ff)
    assert rel_err(ff.cpu().numpy(), ref) < 1e-5
    # back to Kantor: the module's default forces again
    mod.set_bending("kantor")
    ff.zero_()
    mod.apply(C.RbcParams(**par), dev(pp), ff)
    assert rel_err(ff.cpu().numpy(), oracle.rbc_forces(F, nv, pp, par, mode=0)) < 1e-5
    assert C.device_error() == 0


def test_sim_step_with_juelicher_vs_oracle():
    """The fused step with Juelicher bending against the oracle's composition
    of the reference's modules, one step at a time; the bending survives graph
    capture and goes back to Kantor with a new membrane set."""
    import ctc_b200 as C
    L = (16, 16, 16)
    ps = systems.solvent(L, seed=31)
    pv, tri, par = systems.rbc_system(L, 2, seed=32)
    nv = len(pv) // 2
    dpd = systems.dpd_params()
    fsi = (0.0, 8.0, dpd[2], 0.25)
    sim = C.Sim(L, len(ps), C.DpdParams(*dpd), mass=1.0, dt=systems.DT)
    sim.set_solvent(ps)
    sim.set_membranes(pv, tri, nv, par, C.DpdParams(*fsi), mass=systems.RBC_MASS)
    sim.set_bending("juelicher")
    k0 = oracle.Kiss(0, 0, 0, 0)
    kh = [oracle.Kiss.halo(f) for f in range(26)]
    kf = oracle.Kiss(1908, 1409, 290, 12968)
    rs, rv = ps, pv
    for step in range(2):
        seeds = np.array([k0.get()] + [k.get() for k in kh], np.float32)
        fseeds = (kf.get(), kf.get())
        sim.step(1)
        rs, rv = oracle.rbc_step(L, rs, rv, tri, nv, dpd, fsi, par, seeds, fseeds, None, systems.DT, 1.0,
                                 systems.RBC_MASS, bending="juelicher")
        gs, gv = sim.get_solvent(), sim.get_membranes()
        assert np.abs(gs[:, :3] - rs[:, :3]).max() < 2e-6
        assert np.abs(gs[:, 3:] - rs[:, 3:]).max() < 1e-3
        assert np.abs(gv[:, :3] - rv[:, :3]).max() < 2e-6
        assert np.abs(gv[:, 3:] - rv[:, 3:]).max() < 1e-3
        rs, rv = gs, gv
    # graph replay gives the direct launches' state
    out = []
    for graph in (False, True):
        s2 = C.Sim(L, len(ps), C.DpdParams(*dpd), mass=1.0, dt=systems.DT, rng=C.CTC_RNG_STABLE)
        s2.set_solvent(ps)
        s2.set_membranes(pv, tri, nv, par, C.DpdParams(*fsi), mass=systems.RBC_MASS)
        s2.set_bending("juelicher")
        s2.set_graph(graph)
        s2.step(4)
        out.append(s2.get_membranes())
        s2.close()
    assert np.abs(out[0] - out[1]).max() < 1e-4
    sim.close()
    assert C.device_error() == 0
