"""The FP64 forces of the differentiable rollout's step (the test reference
of the adjoint's gradients, oracle.rollout_forces_f64) against independent
restatements: the solvent pairs against the all-pairs numpy forces of
tests/fp64_rollout.py, the FSI pairs against an all-pairs numpy sum with
the stable keys, the membrane forces against the oracle's double path
(orc_rbc_forces_f64) on the same (float-representable) positions."""
import numpy as np

import oracle
from ctc_b200 import systems

from . import fp64_rollout as R


def test_solvent_forces_match_all_pairs():
    L = (6, 6, 6)
    pp = systems.solvent(L, seed=8).astype(np.float64)
    ids = np.arange(len(pp))
    theta = (systems.A_DPD, systems.GAMMA)
    dpd = systems.dpd_params()
    s = np.sqrt(2.0 * systems.KBT * theta[1] / systems.DT)
    F, _ = oracle.rollout_forces_f64(L, pp, ids, (theta[0], theta[1], s, dpd[3]), 0.375)
    ref = R.forces(np.array(L, float), pp[:, :3], pp[:, 3:], ids, theta, dpd[3], systems.KBT, systems.DT, 0.375)
    assert np.abs(F - ref).max() <= 1e-10 * np.abs(ref).max()


def test_fsi_and_membrane_forces():
    L = (14, 14, 14)
    pp = systems.solvent(L, seed=9).astype(np.float64)
    pv, tri, par = systems.rbc_system(L, 1, seed=10)
    pv = pv.astype(np.float64)
    ids = np.arange(len(pp))
    fsi = (0.0, 8.0, systems.dpd_params()[2], 0.25)
    zero = (0.0, 0.0, 0.0, 1.0)
    F, Fv = oracle.rollout_forces_f64(L, pp, ids, zero, 0.0, pv, fsi, 0.625, tri, 642, par)
    # membranes alone: the oracle's double path on the same positions
    ref_m = oracle.rbc_forces(tri, 642, pv.astype(np.float32), par, f64=True)
    # FSI alone, all pairs by minimum image
    d = pv[:, None, :3] - pp[None, :, :3]
    d -= np.array(L) * np.round(d / np.array(L))
    r2 = (d * d).sum(-1)
    k, j = np.nonzero((r2 < 1.0) & (r2 >= 1e-6))
    dd = d[k, j]
    r = np.sqrt(r2[k, j])
    e = dd / r[:, None]
    ev = (e * (pv[k, 3:] - pp[j, 3:])).sum(1)
    w = 1.0 - r
    wr = w ** fsi[3]
    rnd = oracle.mean0var1_batch(np.float32(0.625), k.astype(np.uint32), j.astype(np.uint32), unsigned=True)
    phi = (-fsi[1] * wr * ev + fsi[2] * rnd.astype(np.float64)) * wr + fsi[0] * w
    fv = np.zeros_like(Fv)
    fs = np.zeros_like(F)
    np.add.at(fv, k, phi[:, None] * e)
    np.add.at(fs, j, -phi[:, None] * e)
    assert len(k) > 1000
    assert np.abs(Fv - (fv + ref_m)).max() <= 1e-9 * np.abs(ref_m).max()
    assert np.abs(F - fs).max() <= 1e-10 * np.abs(fs).max()
