"""CPU checks of the oracle's membrane restatement (no GPU): adjacency of the
reference's 642-vertex cell, and forces that are the negative gradient of
the bending energy and of the area/volume/spring energies."""
import os

import numpy as np

import oracle
from ctc_b200 import mesh, systems

from .conftest import GOLDEN


def test_adjacency_642():
    V, F = mesh.read_off(os.path.join(GOLDEN, "rbc.642.off"))
    md, a0, a1 = oracle.adj_build(F, len(V))
    assert md == 6
    val = (a0.reshape(-1, 6) >= 0).sum(1)
    assert sorted(np.bincount(val).tolist())[-2:] == [12, 630]   # valence 5: 12, 6: 630


def test_template_topology():
    X, F = mesh.rbc_template()
    assert X.shape == (642, 3) and F.shape == (1280, 3)
    md, a0, a1 = oracle.adj_build(F, 642)
    assert md == 6
    A, V = mesh.area_volume(X, F)
    assert A > 0 and V > 0
    # Evans-Fung thickness: about 0.8 at the centre, about 2.6 at most
    assert abs(X[:, 0].max() - X[:, 0].min() - 7.82) < 0.05
    assert 2.3 < X[:, 2].max() - X[:, 2].min() < 2.7


def test_bending_force_is_energy_gradient():
    V, F = mesh.read_off(os.path.join(GOLDEN, "rbc.642.off"))
    rng = np.random.default_rng(0)
    pp = np.zeros((len(V), 6), np.float32)
    pp[:, :3] = V + rng.normal(0, 0.05, V.shape)
    par = dict(gammaC=0.0, gammaT=0.0, kBT=0.0, kb=1.0, phi=0.0, ks=0.0, x0=0.457, mpow=2.0, ka=0.0, kd=0.0,
               kv=0.0, totArea=1.0, totVolume=1.0)
    f = oracle.rbc_forces(F, len(V), pp, par, f64=True)
    h = 1e-3
    for i in rng.choice(len(V), 5, replace=False):
        for c in range(3):
            p1, p2 = pp.copy(), pp.copy()
            p1[i, c] += h
            p2[i, c] -= h
            g = (oracle.kantor_energy(F, len(V), p1, 1.0) - oracle.kantor_energy(F, len(V), p2, 1.0)) / \
                (float(p1[i, c]) - float(p2[i, c]))
            assert abs(-g - f[i, c]) < 2e-3 * max(1.0, abs(f[i, c])), (i, c, -g, f[i, c])


def test_juelicher_oracle_invariants():
    """The oracle's Juelicher bending (src/rbc/force/bending/juelicher):
    translation invariant and rotation covariant; one dihedral per edge; not
    momentum-free, as the reference's own force_area applies each vertex's
    coefficient to its own area derivative only (not an exact gradient)."""
    from oracle import refkern
    V, F = mesh.read_off(os.path.join(GOLDEN, "rbc.642.off"))
    assert len(refkern.dihedrals(F)) == 3 * len(F) // 2
    rng = np.random.default_rng(1)
    pp = np.zeros((len(V), 6), np.float32)
    pp[:, :3] = V + rng.normal(0, 0.05, V.shape)
    f = oracle.juelicher_forces(F, len(V), pp)
    scale = np.abs(f).max()
    assert scale > 1
    sh = pp.copy()
    sh[:, :3] += np.float32(1.0)
    assert np.abs(oracle.juelicher_forces(F, len(V), sh) - f).max() < 1e-5 * scale
    R = mesh.random_rotation(rng)
    pr = pp.copy()
    pr[:, :3] = (pp[:, :3].astype(np.float64) @ R.T).astype(np.float32)
    assert np.abs(oracle.juelicher_forces(F, len(V), pr) - f @ R.T).max() < 1e-5 * scale
    # two cells: each cell's forces are its own
    two = np.concatenate([pp, sh])
    f2 = oracle.juelicher_forces(F, len(V), two)
    assert np.abs(f2[:len(V)] - f).max() < 1e-12 * scale
    assert 1e-6 < np.abs(f.sum(0)).max() / np.abs(f).sum() < 1e-2


def test_rbc_simple_file_not_determined_by_its_inputs():
    """The reference's disabled rbc.u.simple output (src/test/rbc/u/simple: two
    642-vertex cells, the template moved by the whole-number shifts of its
    initial condition data/ic/two and the 16^3 box; positions and forces
    printed x 0.1 through uscale 0.1).  Rebuilt from the template, the inputs
    equal the printed positions to their digits.  On them the oracle gives
    both cells the same forces (to 1e-3 of the largest: the volume term sees
    absolute positions); the file's two cells differ by almost 3 % -- more
    than the oracle differs from either of them -- so the file's forces are not
    a function of its inputs, and the oracle stays within 5 % of them."""
    import os
    from ctc_b200 import mesh
    from .conftest import GOLDEN
    d = np.loadtxt(os.path.join(GOLDEN, "forces.ref.rbc.u.simple.txt")) * 10.0
    V, F = mesh.read_off(os.path.join(GOLDEN, "rbc.642.off"))
    nv = len(V)
    pp = np.zeros((len(d), 6), np.float32)
    pp[:nv, :3] = V.astype(np.float32) + np.float32(-8)
    pp[nv:, :3] = V.astype(np.float32) + np.array([-7, -6, -5], np.float32)
    assert np.abs(pp[:, :3] - d[:, :3]).max() < 1e-4           # to the printed digits
    A, Vol = mesh.area_volume(V, F)
    par = dict(gammaC=30.0, gammaT=90.0, kBT=0.0444, kb=17.78, phi=6.97, ks=14.8, x0=0.5, mpow=2.0, ka=2450.0,
               kd=100.0, kv=3750.0, totArea=A, totVolume=Vol)
    f = oracle.rbc_forces(F, nv, pp, par, f64=True)
    ff = d[:, 3:]
    fmax = np.abs(ff).max()
    assert np.abs(f[:nv] - f[nv:]).max() / fmax < 1e-3
    file_cells = np.abs(ff[:nv] - ff[nv:]).max() / fmax
    assert file_cells > 2e-2
    assert np.abs(f - ff).max() / fmax < min(0.05, file_cells)
