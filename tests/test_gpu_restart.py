"""Restart files of the whole step (flu_strt_dump / rbc_strt_dump,
src/flu/imp/start.h and src/rbc/imp/start.h): a run dumped after some steps
and restarted from its files continues as the run itself does.  The random
pair force is off (sigma = 0) because, as in the reference, the generators'
trunks are not part of the restart files."""
import numpy as np
import pytest

import ctc_b200 as C
from ctc_b200 import systems

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _sim(L, ps, pv, tri, nv, par):
    dpd = systems.dpd_params()
    sim = C.Sim(L, len(ps) + 1000, C.DpdParams(dpd[0], dpd[1], 0.0, dpd[3]), mass=1.0, dt=systems.DT)
    sim.set_solvent(ps)
    sim.set_membranes(pv, tri, nv, par, C.DpdParams(0.0, 8.0, 0.0, 0.25), mass=systems.RBC_MASS)
    return sim


def test_sim_restart_continues_the_run(tmp_path):
    L = (16, 16, 16)
    ps = systems.solvent(L, seed=41)
    pv, tri, par = systems.rbc_system(L, 2, seed=42)
    nv = len(pv) // 2
    a = _sim(L, ps, pv, tri, nv, par)
    a.step(3)
    a.strt_dump(tmp_path, 3)
    ps3 = C.restart_read_pp(tmp_path, "flu.pp", 3)
    pv3 = C.restart_read_pp(tmp_path, "rbc.pp", 3)
    assert np.array_equal(ps3, a.get_solvent()) and np.array_equal(pv3, a.get_membranes())
    b = _sim(L, ps3, pv3, tri, nv, par)
    a.step(2)
    b.step(2)
    sa, sb = a.get_solvent(), b.get_solvent()
    assert len(sa) == len(sb) == len(ps)
    assert np.abs(sa - sb).max() < 1e-5
    assert np.abs(a.get_membranes() - b.get_membranes()).max() < 1e-5
    a.close()
    b.close()
    assert C.device_error() == 0
