"""The oracle's membrane-membrane contact (src/cnt) on the CPU: the DPD + LJ
pair against the closed form of src/pair/dev.h:49-75, and the conservation of
momentum of the bulk and periodic-image pairs."""
import numpy as np

import oracle
from ctc_b200 import systems

LJ = (0.3, 0.44)                         # ljs, lje of src/test/contact/0/conf.cfg


def test_lj_closed_form():
    """a = g = s = 0: the force is the capped LJ magnitude along e."""
    p = (0.0, 0.0, 0.0, 0.25) + LJ
    for r in (0.2, 0.25, 0.3, 0.33, 0.336, 0.5, 0.99):
        f = oracle.pair_force_dpdlj(p, [r, 0, 0, 0, 0, 0], [0] * 6, 0.0)
        t6 = (LJ[0] / r) ** 6
        ref = min(max(24 * LJ[1] / r * t6 * (2 * t6 - 1), 0.0), 1e4)
        assert abs(f[0] - ref) <= 1e-5 * max(1.0, ref), (r, f[0], ref)
        assert f[1] == 0 and f[2] == 0
    # beyond the cutoff: nothing; at the cap
    assert not oracle.pair_force_dpdlj(p, [1.0, 0, 0, 0, 0, 0], [0] * 6, 0.0).any()
    assert oracle.pair_force_dpdlj(p, [0.1, 0, 0, 0, 0, 0], [0] * 6, 0.0)[0] == 1e4


def test_dpd_part_is_the_solvent_pair():
    """ljs = 0: the DPD part equals the plain DPD pair force."""
    d = systems.dpd_params()
    rng = np.random.default_rng(3)
    for _ in range(20):
        pa = np.concatenate([rng.uniform(-0.5, 0.5, 3), rng.normal(0, 0.2, 3)]).astype(np.float32)
        pb = np.concatenate([rng.uniform(-0.5, 0.5, 3), rng.normal(0, 0.2, 3)]).astype(np.float32)
        r = float(rng.normal())
        assert np.array_equal(oracle.pair_force_dpdlj(tuple(d) + (0.0, 0.0), pa, pb, r),
                              oracle.pair_force(d, pa, pb, r))


def test_contact_conserves_momentum():
    """Two overlapping membranes, one across the +x face: every pair (bulk,
    and each image against a local vertex) gives +f and -f."""
    L = (16, 12, 14)
    pv, tri, par = systems.rbc_system(L, 1, seed=11)
    nv = len(pv)
    pv2 = pv.copy()
    pv2[:, 2] += 0.8
    pv = np.concatenate([pv, pv2])
    pv[:nv, 0] += L[0] / 2 - pv[:nv, 0].max() + 0.7
    p = tuple(systems.dpd_params()[:3]) + (0.25,) + LJ
    fv = oracle.cnt_forces(L, pv, p, 0.37, 0.71).astype(np.float64)
    assert np.abs(fv).max() > 1.0
    assert np.abs(fv.sum(0)).max() < 1e-5 * np.abs(fv).sum()
    assert len(oracle.fsi_halo_images(L, pv)[0]) > 0
