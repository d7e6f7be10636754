"""Membrane-membrane contact (src/cnt) on the device against the oracle: the
module entry point (bulk + periodic images, seeded and drawing the reference's
trunk) and the fused step with contact switched on.

Tolerance as for the other pair forces against the CPU oracle: per-vertex
max-norm error relative to the vertex's force (floored at 0.1 x the mean),
below 2e-3 for all vertices (the device's rsqrtf/powf are the reference's
fast-math instructions, the oracle's correctly rounded libm ones)."""
import numpy as np
import pytest

import oracle
from ctc_b200 import systems

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

LJ = (0.3, 0.44)                         # ljs, lje of src/test/contact/0/conf.cfg


def dev(x):
    return torch.as_tensor(np.ascontiguousarray(x), device="cuda")


def rel_err(f, ref):
    f = np.asarray(f, np.float64).reshape(-1, 3)
    ref = np.asarray(ref, np.float64).reshape(-1, 3)
    mag = np.abs(ref).max(1)
    return float((np.abs(f - ref).max(1) / np.maximum(mag, 0.1 * mag.mean())).max())


def _membranes(L, seed, gap=0.8):
    """Two copies of a cell, the second shifted by gap along z (the membranes
    overlap: LJ and DPD pairs between them), the first across the +x face."""
    pv, tri, par = systems.rbc_system(L, 1, seed=seed)
    nv = len(pv)
    pv2 = pv.copy()
    pv2[:, 2] += gap
    pv = np.concatenate([pv, pv2])
    pv[:nv, 0] += L[0] / 2 - pv[:nv, 0].max() + 0.7
    return pv, tri, nv, par


def _params():
    d = systems.dpd_params()
    return (d[0], d[1], d[2], 0.25) + LJ


@pytest.mark.parametrize("L,gap", [((16, 16, 16), 0.8), ((12, 10, 14), 0.8), ((16, 16, 16), 0.25)])
def test_contact_vs_oracle(L, gap):
    """gap 0.8: DPD pairs between the membranes; gap 0.25: the LJ repulsion
    too (pairs closer than 2^(1/6) ljs)."""
    import ctc_b200 as C
    pv, tri, nv, par = _membranes(L, seed=21, gap=gap)
    p = _params()
    ref = oracle.cnt_forces(L, pv, p, 0.31, 0.67)
    fv = torch.zeros((len(pv), 3), device="cuda")
    C.Contact(L, len(pv)).apply_seeded(C.DpdLjParams(*p), dev(pv), 0.31, 0.67, fv)
    assert C.device_error() == 0
    assert len(oracle.fsi_halo_images(L, pv)[0]) > 0
    f = fv.cpu().numpy()
    assert rel_err(f, ref) < 2e-3
    assert abs(fv.double().sum().item()) < 1e-4 * fv.abs().sum().item()


def test_contact_module_draws_reference_seeds():
    import ctc_b200 as C
    L = (14, 14, 14)
    pv, tri, nv, par = _membranes(L, seed=23)
    p = _params()
    k = oracle.Kiss(7119, 187, 18278, 15674)
    mod = C.Contact(L, len(pv))
    for _ in range(2):
        sb, sh = k.get(), k.get()
        ref = oracle.cnt_forces(L, pv, p, sb, sh)
        fv = torch.zeros((len(pv), 3), device="cuda")
        mod.apply(C.DpdLjParams(*p), dev(pv), fv)
        assert rel_err(fv.cpu().numpy(), ref) < 2e-3


def test_sim_step_with_contact_vs_oracle():
    """The fused step with contact against the oracle's composition of the
    reference's modules, one step at a time."""
    import ctc_b200 as C
    L = (16, 16, 16)
    ps = systems.solvent(L, seed=25)
    pv, tri, nv, par = _membranes(L, seed=26)
    dpd = systems.dpd_params()
    fsi = (0.0, 8.0, dpd[2], 0.25)
    p = _params()
    sim = C.Sim(L, len(ps), C.DpdParams(*dpd), mass=1.0, dt=systems.DT)
    sim.set_solvent(ps)
    sim.set_membranes(pv, tri, nv, par, C.DpdParams(*fsi), mass=systems.RBC_MASS)
    sim.set_contact(C.DpdLjParams(*p))
    k0 = oracle.Kiss(0, 0, 0, 0)
    kh = [oracle.Kiss.halo(f) for f in range(26)]
    kf = oracle.Kiss(1908, 1409, 290, 12968)
    kc = oracle.Kiss(7119, 187, 18278, 15674)
    rs, rv = ps, pv
    for step in range(2):
        seeds = np.array([k0.get()] + [k.get() for k in kh], np.float32)
        fseeds = (kf.get(), kf.get())
        cseeds = (kc.get(), kc.get())
        sim.step(1)
        rs, rv = oracle.rbc_step(L, rs, rv, tri, nv, dpd, fsi, par, seeds, fseeds, None, systems.DT, 1.0,
                                 systems.RBC_MASS, cnt=p, cnt_seeds=cseeds)
        gs, gv = sim.get_solvent(), sim.get_membranes()
        assert np.abs(gs[:, :3] - rs[:, :3]).max() < 2e-6
        assert np.abs(gs[:, 3:] - rs[:, 3:]).max() < 1e-3
        assert np.abs(gv[:, :3] - rv[:, :3]).max() < 2e-6
        assert np.abs(gv[:, 3:] - rv[:, 3:]).max() < 1e-3
        rs, rv = gs, gv
    sim.set_contact(None)                # and off again
    sim.step(1)
    assert C.device_error() == 0
