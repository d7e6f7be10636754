"""GPU parity of the membrane forces and the solvent-membrane (FSI) forces
against the CPU oracle, through the C ABI."""
import os

import numpy as np
import pytest

import oracle
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


def _cells(nc, seed, template="642.off"):
    if template == "642.off":
        V, F = mesh.read_off(os.path.join(GOLDEN, "rbc.642.off"))
    else:
        V, F = mesh.rbc_template()
    rng = np.random.default_rng(seed)
    r = np.concatenate([V @ mesh.random_rotation(rng).T + rng.uniform(-5, 5, 3) for _ in range(nc)])
    r += rng.normal(0, 0.02, r.shape)          # off equilibrium
    pp = np.zeros((len(r), 6), np.float32)
    pp[:, :3] = r
    pp[:, 3:] = rng.normal(0, 0.3, (len(r), 3))
    A, Vol = mesh.area_volume(V, F)
    return pp, F, len(V), systems.rbc_params(A * 1.01, Vol * 0.99)


@pytest.mark.parametrize("template", ["642.off", "evans-fung"])
def test_membrane_forces_vs_oracle(template):
    import ctc_b200 as C
    pp, F, nv, par = _cells(3, 1, template)
    ref = oracle.rbc_forces(F, nv, pp, par, mode=0)
    mod = C.RbcForce(F, nv, 8)
    assert mod.md == oracle.mesh_md(F, nv)
    ff = torch.zeros((len(pp), 3), device="cuda")
    mod.apply(C.RbcParams(**par), dev(pp), ff)
    assert C.device_error() == 0
    assert rel_err(ff.cpu().numpy(), ref) < 1e-5
    av = mod.area_volume(dev(pp)).cpu().numpy()
    assert np.allclose(av, oracle.area_volume(F, nv, pp), rtol=1e-12)
    # error statement against all-double arithmetic
    ref64 = oracle.rbc_forces(F, nv, pp, par, f64=True)
    assert rel_err(ff.cpu().numpy(), ref64) < 1e-4


def test_membrane_bending_off():
    import ctc_b200 as C
    pp, F, nv, par = _cells(2, 2)
    par0 = dict(par, kb=0.0)
    ref = oracle.rbc_forces(F, nv, pp, par0, mode=0)
    mod = C.RbcForce(F, nv, 2)
    mod.set_bending(False)
    ff = torch.zeros((len(pp), 3), device="cuda")
    mod.apply(C.RbcParams(**par), dev(pp), ff)
    assert rel_err(ff.cpu().numpy(), ref) < 1e-5


def test_membrane_momentum_free():
    """internal forces of a cell at rest sum to zero (translation invariance of
    every term but the per-triangle volume term, which sums to zero per cell)"""
    import ctc_b200 as C
    pp, F, nv, par = _cells(1, 3)
    pp[:, 3:] = 0
    mod = C.RbcForce(F, nv, 1)
    ff = torch.zeros((len(pp), 3), device="cuda", dtype=torch.float32)
    mod.apply(C.RbcParams(**par), dev(pp), ff)
    f = ff.double().cpu().numpy()
    assert np.abs(f.sum(0)).max() < 1e-4 * np.abs(f).sum()


@pytest.mark.parametrize("L", [(16, 16, 16), (12, 10, 14)])
def test_fsi_vs_oracle(L):
    import ctc_b200 as C
    ps0 = systems.solvent(L, seed=5)
    counts, starts, order, ps = oracle.clist_build(L, ps0)
    pv, F, par = systems.rbc_system(L, 2, seed=6)
    # push one cell across the +x face so that periodic images interact
    nv = len(pv) // 2
    pv[:nv, 0] += L[0] / 2 - pv[:nv, 0].max() + 1.5
    dpd = (0.0, 8.0, systems.dpd_params()[2], 0.25)       # a = 0, gamma = 8
    fv_ref, fs_ref = oracle.fsi_forces(L, pv, ps, starts, dpd, 0.25, 0.75)
    fv = torch.zeros((len(pv), 3), device="cuda")
    fs = torch.zeros((len(ps), 3), device="cuda")
    C.Fsi(L, len(pv), len(ps)).apply_seeded(C.DpdParams(*dpd), dev(pv), dev(ps), dev(starts), dev(counts), 0.25,
                                            0.75, fv, fs)
    assert C.device_error() == 0
    assert len(oracle.fsi_halo_images(L, pv)[0]) > 0
    assert rel_err(fv.cpu().numpy(), fv_ref) < 2e-3
    assert rel_err(fs.cpu().numpy(), fs_ref) < 2e-3
    # total momentum exchange balances
    assert abs(fv.double().sum().item() + fs.double().sum().item()) < 1e-3 * fv.abs().sum().item()


def test_fsi_module_draws_reference_seeds():
    import ctc_b200 as C
    L = (12, 12, 12)
    counts, starts, order, ps = oracle.clist_build(L, systems.solvent(L, seed=7))
    pv, F, par = systems.rbc_system(L, 1, seed=8)
    dpd = (0.0, 8.0, systems.dpd_params()[2], 0.25)
    k = oracle.Kiss(1908, 1409, 290, 12968)
    mod = C.Fsi(L, len(pv), len(ps))
    for _ in range(2):
        sb, sh = k.get(), k.get()
        fv_ref, fs_ref = oracle.fsi_forces(L, pv, ps, starts, dpd, sb, sh)
        fv = torch.zeros((len(pv), 3), device="cuda")
        fs = torch.zeros((len(ps), 3), device="cuda")
        mod.apply(C.DpdParams(*dpd), dev(pv), dev(ps), dev(starts), dev(counts), fv, fs)
        assert rel_err(fv.cpu().numpy(), fv_ref) < 2e-3
