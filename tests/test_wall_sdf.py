"""The host side of the walls (no GPU): the field file read, scaled and
resampled onto the texture grid (sdf_gen, src/wall/sdf/imp/gen.h) by this
build, by the oracle and by the reference's own host code compiled from its
sources (oracle/_ref/librefsdf.so via oracle/ref.mk) -- bit for bit, with the
same grid transform and far threshold; and the oracle's freezing."""
import ctypes
import os

import numpy as np
import pytest

import oracle
import ctc_b200 as C

from .conftest import GOLDEN

SDF = os.path.join(GOLDEN, "sdf")
REFSDF = os.path.join(os.path.dirname(oracle.__file__), "_ref", "librefsdf.so")


def _ref_texture(path, L):
    lib = ctypes.CDLL(REFSDF)
    T, o, s = (ctypes.c_int * 3)(), (ctypes.c_float * 3)(), (ctypes.c_float * 3)()
    lib.refsdf_texture(path.encode(), *L, T, None, o, s)
    tex = np.zeros(T[0] * T[1] * T[2], np.float32)
    lib.refsdf_texture(path.encode(), *L, T, tex.ctypes.data_as(ctypes.c_void_p), o, s)
    return list(T), tex, np.array(o[:], np.float32), np.array(s[:], np.float32)


@pytest.mark.parametrize("name,L", [("yplates.dat", (16, 16, 16)), ("wall.dat", (16, 12, 20))])
def test_texture_matches_reference_host_code(name, L):
    path = os.path.join(SDF, name)
    N, ext, D = C.sdf_read(path)
    T, tex, o, s, thr = C.sdf_resample(N, ext, D, L)
    q = oracle.Sdf(N, ext, D, L)
    assert T == list(q.T)
    assert np.array_equal(tex.reshape(-1).view(np.uint32), q.tex.view(np.uint32))
    assert np.array_equal(o, q.o) and np.array_equal(s, q.s) and np.float32(thr) == q.thr[0]
    if not os.path.exists(REFSDF):
        pytest.skip("oracle/_ref/librefsdf.so not built")
    rT, rtex, ro, rs = _ref_texture(path, L)
    assert rT == T
    assert np.array_equal(tex.reshape(-1).view(np.uint32), rtex.view(np.uint32))
    assert np.array_equal(o, ro) and np.array_equal(s, rs)


def test_oracle_freeze_plates():
    """Freezing a uniform solvent against the z plates of wall.dat: the wall
    layer has the density of the solvent, its images fill the margin, and
    no bulk particle is inside the wall."""
    path = os.path.join(SDF, "wall.dat")
    L = (16, 16, 16)
    q = oracle.Sdf(*oracle.sdf_read(path), L)
    rng = np.random.default_rng(0)
    n = 10 * 16 ** 3
    pp = np.zeros((n, 6), np.float32)
    pp[:, :3] = rng.uniform(-8, 8, (n, 3))
    s = q.eval(pp)
    bulk, wpos, ws = q.freeze(pp)
    assert len(bulk) == int((s < 0).sum())
    assert (q.eval(bulk) < 0).all()
    nwall = int(((s >= 0) & (s <= 2)).sum())
    assert len(wpos) > nwall            # the images in the margin
    assert ws[-1] == len(wpos)
    LW = np.array(L) + 12
    cell = np.floor(wpos[:, :3].astype(np.float64) + LW // 2).astype(np.int64)
    cid = cell[:, 0] + LW[0] * (cell[:, 1] + LW[1] * cell[:, 2])
    assert (np.diff(cid) >= 0).all()    # cell-sorted
    assert np.array_equal(np.bincount(cid, minlength=int(np.prod(LW))), np.diff(ws))
