"""The oracle's membrane pieces pinned to the reference's own host code, built
from its sources into oracle/_ref/librefhost.so by oracle/ref.mk: the ring
adjacency of adj_ini (src/rbc/adj/imp/ini.h, src/algo/edg) and the FP64 host
build of the Kantor dihedral forces (src/mesh/force/kantor0/imp.cpp), walked
over every (vertex, ring slot) as kantor_dev::force walks them.

Tolerances: adjacency tables bit-exact; Kantor forces within 1e-12 relative
(max-norm per vertex) with no spontaneous angle: both sides are FP64 from the
same float positions, the reference's host build with pow(x, -0.5) for the
reciprocal square roots where the oracle takes 1 / sqrt(x).  With a
spontaneous angle the term sin(phi) / sin(theta) of near-flat dihedrals
(1 - cos^2 theta a difference of nearly equal numbers) amplifies that last-bit
difference: 1e-9 there."""
import os

import numpy as np
import pytest

import oracle
from ctc_b200 import mesh, systems
from oracle import refkern

from .conftest import GOLDEN

pytestmark = pytest.mark.skipif(not refkern.host_available(), reason="oracle/_ref/librefhost.so not built")


def _templates():
    out = []
    for name in ("rbc.642.off", "rbc.1986.off", "rbc.2562.off"):
        V, F = mesh.read_off(os.path.join(GOLDEN, name))
        out.append((name, V, F))
    V, F = mesh.rbc_template()
    out.append(("evans-fung", V, F))
    return out


@pytest.mark.parametrize("name,V,F", _templates(), ids=[t[0] for t in _templates()])
def test_adjacency_equals_reference_adj_ini(name, V, F):
    md, a0, a1 = oracle.adj_build(F, len(V))
    r0, r1 = refkern.host_adj(F, len(V), md)
    assert np.array_equal(a0, r0) and np.array_equal(a1, r1)


def rel_err(f, ref):
    f = np.asarray(f, np.float64).reshape(-1, 3)
    ref = np.asarray(ref, np.float64).reshape(-1, 3)
    mag = np.abs(ref).max(1)
    return float((np.abs(f - ref).max(1) / np.maximum(mag, 0.1 * mag.mean())).max())


@pytest.mark.parametrize("phi", [0.0, 6.97])
def test_oracle_kantor_forces_equal_reference_host_build(phi):
    """Bending alone (every other membrane constant zero) on three perturbed
    cells of the configurations' template, with the spontaneous angle off and
    on."""
    V, F = mesh.rbc_template()
    rng = np.random.default_rng(11)
    nc = 3
    r = np.concatenate([V @ mesh.random_rotation(rng).T + rng.uniform(-5, 5, 3) for _ in range(nc)])
    r += rng.normal(0, 0.03, r.shape)
    pp = np.zeros((len(r), 6), np.float32)
    pp[:, :3] = r
    kb = 40 * systems.KBT
    par = dict(gammaC=0.0, gammaT=0.0, kBT=systems.KBT, kb=kb, phi=phi, ks=0.0, x0=0.457, mpow=2.0, ka=0.0, kd=0.0,
               kv=0.0, totArea=1.0, totVolume=1.0)
    got = oracle.rbc_forces(F, len(V), pp, par, f64=True)
    md = oracle.mesh_md(F, len(V))
    # RbcParams holds kb and phi as floats (src/rbc/params/type.h)
    ref = refkern.host_kantor(F, len(V), md, pp, float(np.float32(kb)), float(np.float32(phi)))
    assert np.abs(ref).max() > 1e-3
    assert rel_err(got, ref) < (1e-12 if phi == 0 else 1e-9)
