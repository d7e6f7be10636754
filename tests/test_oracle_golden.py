"""Pins the CPU oracle to the reference's own golden vectors and known answers.

Golden files come from the reference's test suite (src/test_data, copied by
tests/golden/make_fixtures.py); the tests that produce them are the active
``# TEST:`` scripts src/test/rnd/main, src/test/clist/{0,1,2}/main,
src/test/pair/0/main and src/test/rbc/u/area_volume/dev/main.
"""
import os

import numpy as np
import pytest

import oracle
from ctc_b200 import mesh

from .conftest import GOLDEN


def _lines(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return [l.rstrip("\n") for l in f if l.strip()]


def test_kiss_rnd_t0():
    """src/test/rnd/main: KISS(42,42,42,42), 100 draws printed with %10.6e."""
    k = oracle.Kiss(42, 42, 42, 42)
    got = ["%10.6e" % k.get() for _ in range(100)]
    assert got == _lines("rnd.ref.rnd.t0.txt")


def test_bulk_trunk_degenerates_to_lcg():
    """rnd_ini(0,0,0,0) (src/fluforces/imp/ini.h:6): y = z = c = 0 stay 0, the
    seed sequence is x_k / 2^32 with x_{k+1} = 69069 x_k + 12345 mod 2^32."""
    k = oracle.Kiss(0, 0, 0, 0)
    x = 0
    for _ in range(1000):
        x = (69069 * x + 12345) & 0xFFFFFFFF
        assert k.get() == float(np.float32(np.float32(x) / np.float32(2 ** 32)))


def _read_pa(line):
    t = line.split()
    return [float(v) for v in t[:6]], t[6], t[7]


def test_halo_trunks_pairwise():
    """Known answer of the halo trunk seeding (src/fluforces/imp/ini.h:22-59
    on a 1-rank periodic cart): fragment f and its anti-fragment start from
    the same KISS state, so both sides of a pair across a face draw the same
    random number -- except the edges (-1, 0, 1) and (1, 0, -1), whose
    "plus" rule picks opposite signs (seeds 21 and 5): pairs across that edge
    get a different random force on each side, so the halo pairs cannot be
    evaluated once per pair with the reaction given to the other side."""
    odd = []
    for f in range(26):
        a = oracle.frag_anti(f)
        kf, ka = oracle.Kiss.halo(f), oracle.Kiss.halo(a)
        if any(kf.get() != ka.get() for _ in range(4)):
            odd.append(oracle.frag_dir(f))
    assert sorted(odd) == [(-1, 0, 1), (1, 0, -1)]


def test_pair_0():
    """src/test/pair/0: pairs of src/data/pair/2 with a = 2.6666667, g = 8,
    spow = 0.25 and RND unset (0); every pair here uses the DPD view (the LJ
    one is only taken for SOLID-SOLID, src/u/pair/imp/main.h:14-43)."""
    lines = _lines("pair.in.2.txt")
    expect = _lines("pair.ref.pair.0.txt")
    got = []
    for la, lb in zip(lines[0::2], lines[1::2]):
        pa, ka, _ = _read_pa(la)
        pb, kb, _ = _read_pa(lb)
        assert not (ka == "SOLID" and kb == "SOLID")
        f = oracle.pair_force((2.6666667, 8.0, 0.0, 0.25), pa, pb, 0.0)
        got.append("%g %g %g" % tuple(float(x) for x in f))
    assert got == expect


@pytest.mark.parametrize("case", ["t0", "t1", "t2"])
def test_clist_golden(case):
    """src/test/clist/{0,1,2}: box 4x6x8, particles from pre/units/gen_random;
    output: validity flag, then start and count of every cell."""
    L = (4, 6, 8)
    pp = oracle.read_floats(os.path.join(GOLDEN, "clist.in.%s.txt" % case)).reshape(-1, 6)
    counts, starts, order, out = oracle.clist_build(L, pp)
    # validity check of src/u/clist/main.cu:74-110 on the sorted output
    ok = True
    for cid in range(L[0] * L[1] * L[2]):
        cx, cy, cz = cid % 4, (cid // 4) % 6, cid // 24
        for j in range(starts[cid], starts[cid] + counts[cid]):
            r = out[j]
            for c, d, x in ((cx, 4, r[0]), (cy, 6, r[1]), (cz, 8, r[2])):
                ok &= bool((x >= c - 0.5 * d) and (x < c + 1 - 0.5 * d))
    got = ["0" if ok else "1"]
    for cid in range(L[0] * L[1] * L[2]):
        got += [str(starts[cid]), str(counts[cid])]
    assert got == _lines("clist.ref.clist.%s.txt" % case)


def test_area_volume_1986():
    """src/test/rbc/u/area_volume/dev: 1986-vertex cell, identity placement,
    printed with %g: 944.577 1753.5."""
    V, F = mesh.read_off(os.path.join(GOLDEN, "rbc.1986.off"))
    pp = np.zeros((len(V), 6), np.float32)
    pp[:, :3] = V
    ref = [float(x) for x in _lines("av.ref.rbc.u.area_volume.dev.0.txt")[0].split()]
    av64 = oracle.area_volume(F, len(V), pp)[0]
    av32 = oracle.area_volume(F, len(V), pp, f32=True)[0]
    # the reference sums floats in warp-reduce + atomic order; the exact sum
    # prints as the golden line, a sequential float sum is within 2e-6
    assert "%g %g" % (av64[0], av64[1]) == "%g %g" % tuple(ref)
    assert np.allclose(av32, av64, rtol=2e-6)


def test_kantor_angles_eng_kantor():
    """src/test_data/eng.ref.mesh.eng_kantor.txt (src/test/mesh/eng_kantor:
    the 2562-vertex sphere, kb = 1, angle0 = 0): per vertex, the mean over
    its edges of the mesh tool's 2 kb (1 - cos theta)
    (src/mesh/eng_kantor/imp/main.h:22-33, edge-to-vertex average of
    src/mesh/scatter).  The oracle's Kantor dihedral angles reproduce it to
    the file's six printed digits, which pins the angle the bending force
    differentiates."""
    V, F = mesh.read_off(os.path.join(GOLDEN, "rbc.2562.off"))
    pp = np.zeros((len(V), 6), np.float32)
    pp[:, :3] = V
    ev = 2 * oracle.kantor_vertex_energy(F, len(V), pp, 1.0)
    g = np.loadtxt(os.path.join(GOLDEN, "eng.ref.mesh.eng_kantor.txt"))
    assert g.shape == (len(V), 4)
    assert np.abs(ev - g[:, 3]).max() <= 5e-6 * np.abs(g[:, 3]).max()
    assert (np.abs(ev - g[:, 3]) <= 1e-5 * np.abs(g[:, 3]) + 1e-12).all()


# src/test/bulk/{0,1}/main: u/bulk on gen_random particles in a 4^3 box, kBT = 0
# (no random force), a = 2.6666667, g = 8, spow = 0.25 (conf.cfg); the output
# is the sorted particles and their bulk forces, scaled by uscale and sorted as
# text lines
BULK_GOLDEN = {"t0": 1e4, "t1": 1e2}
BULK_DPD = (2.6666667, 8.0, 0.0, 0.25)


def bulk_golden(case):
    """(input particles, golden rows (x y z vx vy vz fx fy fz))."""
    pp = np.loadtxt(os.path.join(GOLDEN, "bulk.in.%s.txt" % case), dtype=np.float32)
    g = np.loadtxt(os.path.join(GOLDEN, "ff.ref.bulk.%s.txt" % case)) / BULK_GOLDEN[case]
    return pp, g


def match_bulk(ppout, ff, g):
    """Per golden row, the relative force error of the particle at its position
    (floored at 0.1 x the mean force)."""
    mags = np.abs(g[:, 6:9]).max(1)
    err = []
    for row, m in zip(g, mags):
        d = np.abs(ppout[:, :3] - row[:3]).sum(1)
        k = int(d.argmin())
        assert d[k] < 1e-3
        err.append(np.abs(ff[k] - row[6:9]).max() / max(m, 0.1 * mags.mean()))
    return max(err)


@pytest.mark.parametrize("case", ["t0", "t1"])
def test_bulk_forces_golden(case):
    """ff.ref.bulk.{t0,t1}: the oracle's bulk forces to the file's digits."""
    pp, g = bulk_golden(case)
    L = (4, 4, 4)
    counts, starts, order, ppout = oracle.clist_build(L, pp)
    assert len(ppout) == len(g)
    ff = oracle.dpd_bulk(L, ppout, starts, BULK_DPD, 0.0)
    assert match_bulk(ppout, ff, g) < 1e-5
