"""bop particle files and restart files (host code, no GPU): the reference's
own bop fixtures (tests/golden/bop, copied by tests/golden/make_bop_fixtures.py
from its post-processing tests) read back, headers written byte for byte as
those files hold them, and the restart / dump naming of src/io/restart and
src/io/bop."""
import os

import numpy as np
import pytest

import ctc_b200 as C

from .conftest import GOLDEN

BOP = os.path.join(GOLDEN, "bop")


def test_read_reference_text_fixtures():
    s = C.bop_read(os.path.join(BOP, "s-00.bop"))
    assert s.dtype == np.float32 and s.shape == (3, 6)
    assert np.array_equal(s, np.array([[0, 0, 0, -1, 2, 3], [1, 0, 0, -1, 2, 3], [0, 1, 0, -1, 2, 3]], np.float32))
    ids = C.bop_read(os.path.join(BOP, "id-00.bop"))
    assert ids.dtype == np.int32 and ids.reshape(-1).tolist() == [0, 1, 2]


def test_header_matches_reference_files(tmp_path):
    """The header the writer makes for the reference's 60,023-particle solvent
    dump and its colours is the reference file's text; the values are the
    records in order (the first 64 of the reference file)."""
    head = np.fromfile(os.path.join(BOP, "solvent-00041.values.head"), np.float32).reshape(64, 6)
    pp = np.zeros((60023, 6), np.float32)
    pp[:64] = head
    C.bop_write(tmp_path / "solvent-00041", pp, "x y z vx vy vz")
    with open(tmp_path / "solvent-00041.bop", "rb") as f, open(os.path.join(BOP, "solvent-00041.bop"), "rb") as g:
        assert f.read() == g.read()
    with open(tmp_path / "solvent-00041.values", "rb") as f:
        data = f.read()
    assert len(data) == 60023 * 24
    with open(os.path.join(BOP, "solvent-00041.values.head"), "rb") as g:
        assert data[:1536] == g.read()
    C.bop_write(tmp_path / "colors_solvent-00041", np.zeros((60023, 1), np.int32), "color")
    with open(tmp_path / "colors_solvent-00041.bop", "rb") as f, \
            open(os.path.join(BOP, "colors_solvent-00041.bop"), "rb") as g:
        assert f.read() == g.read()
    back = C.bop_read(tmp_path / "solvent-00041.bop")
    assert back.shape == (60023, 6) and np.array_equal(back[:64], head)


def test_restart_names_and_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    pp = rng.normal(size=(1000, 6)).astype(np.float32)
    ii = rng.integers(0, 1 << 30, 77).astype(np.int32)
    base = str(tmp_path / "strt")
    C.restart_write_pp(base, "flu.pp", 5, pp)
    C.restart_write_pp(base, "rbc.pp", "final", pp[:642])
    C.restart_write_ii(base, "rbc.ids", "templ", ii)
    assert sorted(os.listdir(tmp_path / "strt")) == ["flu.pp", "rbc.ids", "rbc.pp"]
    assert sorted(os.listdir(tmp_path / "strt" / "flu.pp")) == ["00005.bop", "00005.values"]
    with open(tmp_path / "strt" / "flu.pp" / "00005.bop") as f:
        assert f.read() == "1000\nDATA_FILE: 00005.values\nDATA_FORMAT: float\nVARIABLES: x y z vx vy vz\n"
    with open(tmp_path / "strt" / "rbc.ids" / "templ.bop") as f:
        assert f.read() == "77\nDATA_FILE: templ.values\nDATA_FORMAT: int\nVARIABLES: i\n"
    assert os.path.exists(tmp_path / "strt" / "rbc.pp" / "final.values")
    assert np.array_equal(C.restart_read_pp(base, "flu.pp", 5), pp)
    assert np.array_equal(C.restart_read_pp(base, "rbc.pp", "final"), pp[:642])
    assert np.array_equal(C.restart_read_ii(base, "rbc.ids", "templ"), ii)
    # an empty set, and the errors of a missing file or a file of the wrong kind
    C.restart_write_pp(base, "flu.pp", 0, np.zeros((0, 6), np.float32))
    assert C.restart_read_pp(base, "flu.pp", 0).shape == (0, 6)
    with pytest.raises(C.CtcError):
        C.restart_read_pp(base, "flu.pp", 6)
    with pytest.raises(C.CtcError):
        C.restart_read_pp(base, "rbc.ids", "templ")


def test_io_bop_dumps(tmp_path):
    """io_bop_parts / _forces shift positions to the box's edge, in float;
    ids and colours are int files of one variable."""
    rng = np.random.default_rng(1)
    L = (16, 12, 10)
    pp = rng.uniform(-5, 5, (300, 6)).astype(np.float32)
    ff = rng.normal(size=(300, 3)).astype(np.float32)
    C.io_bop_parts(tmp_path, "solvent", 41, pp, L)
    C.io_bop_parts(tmp_path, "rbc", 41, pp, L, ff=ff)
    C.io_bop_ids(tmp_path, "ids_solvent", 41, np.arange(300))
    C.io_bop_ids(tmp_path, "colors_solvent", 41, np.ones(300), colors=True)
    shifted = pp.copy()
    shifted[:, :3] = np.float32(0.5) * np.asarray(L, np.float32) + pp[:, :3]
    got = C.bop_read(tmp_path / "bop" / "solvent-00041.bop")
    assert np.array_equal(got, shifted)
    got = C.bop_read(tmp_path / "bop" / "rbc-00041.bop")
    assert got.shape == (300, 9) and np.array_equal(got[:, :6], shifted) and np.array_equal(got[:, 6:], ff)
    with open(tmp_path / "bop" / "rbc-00041.bop") as f:
        assert f.read().splitlines()[3] == "VARIABLES: x y z vx vy vz fx fy fz"
    with open(tmp_path / "bop" / "ids_solvent-00041.bop") as f:
        assert f.read().splitlines()[2:] == ["DATA_FORMAT: int", "VARIABLES: ids"]
    with open(tmp_path / "bop" / "colors_solvent-00041.bop") as f:
        assert f.read().splitlines()[3] == "VARIABLES: color"
    assert C.bop_read(tmp_path / "bop" / "colors_solvent-00041.bop").reshape(-1).tolist() == [1] * 300
