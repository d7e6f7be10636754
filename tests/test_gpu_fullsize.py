"""The full benchmark sizes, checked through properties that do not need the
oracle to finish: the 192 x 96 x 96 box of 17.7 M particles and the 64^3 box
with 200 red blood cells.

- cell lists at full size: counts bit-exact against a host recount of the
  reference's cell index (src/clist/dev/main.h:21-24, double precision), and
  every sorted particle inside the cell its start/count range says;
- Newton's third law at full size: with keys symmetric in the two particles
  (stable keys) every pair force enters as +f and -f, so the forces of a
  step sum to zero up to float rounding, and the total momentum of solvent
  and membranes is conserved over steps;
- no particle is lost and no kernel records a failure."""
import ctypes

import numpy as np
import pytest

from ctc_b200 import systems

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

C2 = (192, 96, 96)


def _state(C, sim, n):
    from ctc_b200 import _lib
    pos, vel, force, starts = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
    _lib.check(_lib.lib().ctc_sim_state(sim.h, ctypes.byref(pos), ctypes.byref(vel), ctypes.byref(force),
                                        ctypes.byref(starts)))
    dev = torch.device("cuda")
    nc = sim.L[0] * sim.L[1] * sim.L[2]
    return (C._wrap_dev(pos.value, 4 * n, torch.float32, dev).reshape(n, 4),
            C._wrap_dev(force.value, 4 * n, torch.float32, dev).reshape(n, 4),
            C._wrap_dev(starts.value, nc + 1, torch.int32, dev))


def test_c2_cell_lists_full_size():
    """dt = 0: the state after one step is the cell-sorted input itself."""
    import ctc_b200 as C
    pp = systems.solvent(C2, seed=2)
    n = len(pp)
    sim = C.Sim(C2, n, C.DpdParams(*systems.dpd_params()), dt=0.0)
    sim.set_solvent(pp)
    sim.step(1)
    torch.cuda.synchronize()
    pos, force, starts = _state(C, sim, n)
    Lh = np.asarray(C2) // 2
    # host recount of the reference's cell index, in double
    cell = np.floor(pp[:, :3].astype(np.float64) + Lh).astype(np.int64)
    cid = cell[:, 0] + C2[0] * (cell[:, 1] + C2[1] * cell[:, 2])
    ref_counts = np.bincount(cid, minlength=C2[0] * C2[1] * C2[2])
    st = starts.cpu().numpy().astype(np.int64)
    assert st[-1] == n
    assert np.array_equal(np.diff(st), ref_counts)
    # every sorted particle in the cell its range says
    p = pos[:, :3].double()
    lh = torch.tensor(Lh, dtype=torch.float64, device="cuda")
    c = torch.floor(p + lh).long()
    got = c[:, 0] + C2[0] * (c[:, 1] + C2[1] * c[:, 2])
    want = torch.repeat_interleave(torch.arange(len(st) - 1, device="cuda"),
                                   torch.as_tensor(np.diff(st), device="cuda"))
    assert torch.equal(got, want)
    # the particles are the input's (ids in pos.w)
    ids = pos[:, 3].contiguous().view(torch.int32).long()
    assert torch.equal(torch.sort(ids).values, torch.arange(n, device="cuda"))
    assert C.device_error() == 0
    sim.close()


def test_c2_forces_sum_to_zero_full_size():
    import ctc_b200 as C
    pp = systems.solvent(C2, seed=3)
    n = len(pp)
    sim = C.Sim(C2, n, C.DpdParams(*systems.dpd_params()), rng=C.CTC_RNG_STABLE)
    sim.set_solvent(pp)
    sim.step(2)
    torch.cuda.synchronize()
    pos, force, starts = _state(C, sim, n)
    f = force[:, :3].double()
    assert int(starts[-1].item()) == n
    assert f.abs().sum().item() > 0
    assert f.sum(0).abs().max().item() < 1e-6 * f.abs().sum().item()
    assert C.device_error() == 0
    sim.close()


def test_c3_momentum_conserved_full_size():
    """64^3 solvent + 200 cells, stable keys: solvent-solvent, solvent-membrane
    and the membranes' internal forces all conserve momentum."""
    import ctc_b200 as C
    L = (64, 64, 64)
    ps = systems.solvent(L, seed=4)
    ps[:, 3:] -= ps[:, 3:].mean(0)
    pv, tri, par = systems.rbc_system(L, 200, seed=5)
    pv[:, 3:] = 0.0
    dpd = systems.dpd_params()
    sim = C.Sim(L, len(ps), C.DpdParams(*dpd), rng=C.CTC_RNG_STABLE)
    sim.set_solvent(ps)
    sim.set_membranes(pv, tri, 642, par, C.DpdParams(0.0, 8.0, dpd[2], 0.25), mass=systems.RBC_MASS)
    p0 = ps[:, 3:].astype(np.float64).sum(0)
    sim.step(5)
    gs, gv = sim.get_solvent(), sim.get_membranes()
    assert len(gs) == len(ps) and len(gv) == len(pv)
    p1 = gs[:, 3:].astype(np.float64).sum(0) + systems.RBC_MASS * gv[:, 3:].astype(np.float64).sum(0)
    scale = np.abs(gs[:, 3:]).astype(np.float64).sum()
    assert np.abs(p1 - p0).max() < 1e-6 * scale, (p1 - p0, scale)
    assert C.device_error() == 0
