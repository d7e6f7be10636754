"""Edge cases of the path on the device, as the reference's own checks have
them: an empty solvent, pairs exactly at the cutoff and closer than the
r^2 < 1e-6 guard (src/pair/dev.h:18-21), particles on the box faces and
outside the box (dropped by clist_build without the periodic wrap, wrapped in
the step), a field without a wall, and membranes with no cells."""
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


def test_empty_solvent_steps():
    import ctc_b200 as C
    sim = C.Sim((8, 8, 8), 100, C.DpdParams(*systems.dpd_params()))
    sim.set_solvent(np.zeros((0, 6), np.float32))
    sim.step(3)
    assert sim.get_solvent().shape == (0, 6)
    assert C.device_error() == 0
    sim.close()


def _forces(L, pp, seeds):
    import ctc_b200 as C
    out, starts, counts, ids = C.Clist(L, len(pp)).build(dev(pp))
    ff = torch.zeros((len(pp), 3), device="cuda")
    C.FluForces(L, len(pp)).apply_seeded(C.DpdParams(*systems.dpd_params()), out, starts, counts, seeds, ff)
    c_ref, s_ref, order, ppout = oracle.clist_build(L, pp)
    ref = oracle.dpd_bulk(L, ppout, s_ref, systems.dpd_params(), seeds[0]) + \
        oracle.dpd_halo(L, ppout, s_ref, c_ref, systems.dpd_params(), seeds[1:])
    return ff.cpu().numpy(), ref, ids.cpu().numpy(), order


def test_pairs_at_the_cutoff_and_coincident():
    """r = 1 exactly: no force (r^2 >= 1); r^2 < 1e-6: the direction is zero,
    so the force is zero; both in the bulk and across a periodic face."""
    L = (8, 8, 8)
    pp = np.zeros((8, 6), np.float32)
    pp[0, :3], pp[1, :3] = (0.25, 0.25, 0.25), (1.25, 0.25, 0.25)        # r = 1, same row
    pp[2, :3], pp[3, :3] = (-2.5, 1.5, 1.5), (-2.5, 1.5, 1.5 + 5e-4)      # r^2 = 2.5e-7
    pp[4, :3], pp[5, :3] = (-3.75, -1.5, 0.5), (3.25, -1.5, 0.5)         # r = 1 across the x face
    pp[6, :3], pp[7, :3] = (-3.9999, 2.5, -2.5), (3.9999, 2.5, -2.5)     # r = 2e-4 across the face
    pp[:, 3:] = np.random.default_rng(1).normal(0, 1, (8, 3))
    seeds = np.random.default_rng(2).random(27).astype(np.float32)
    f, ref, ids, order = _forces(L, pp, seeds)
    assert np.array_equal(ids, order)
    assert (f == 0).all() and (ref == 0).all()


def test_particles_on_and_outside_the_faces():
    """clist_build without the wrap drops particles outside [-L/2, L/2)
    (src/clist/dev/main.h:21-41); on the faces they take the first and last
    cells; the step wraps them instead."""
    import ctc_b200 as C
    L = (8, 6, 10)
    rng = np.random.default_rng(3)
    pp = systems.solvent(L, seed=4)[:2000].copy()
    pp[0, :3] = (-4.0, -3.0, -5.0)                                      # the lower faces: cell 0
    pp[1, :3] = (np.nextafter(np.float32(4.0), np.float32(0)), 2.9999, 4.9999)   # just inside the upper faces
    pp[2, :3] = (4.0, 0.0, 0.0)                                        # on the upper x face: outside
    pp[3, :3] = (0.0, -3.5, 0.0)                                       # outside in y
    out, starts, counts, ids = C.Clist(L, len(pp)).build(dev(pp))
    c_ref, s_ref, order, ppout = oracle.clist_build(L, pp)
    assert out.shape[0] == len(pp) - 2 == len(order)
    assert np.array_equal(starts.cpu().numpy(), s_ref)
    assert np.array_equal(ids.cpu().numpy(), order)
    assert 0 in order and 1 in order and 2 not in order and 3 not in order
    # the step wraps the two outside particles back into the box
    sim = C.Sim(L, len(pp), C.DpdParams(*systems.dpd_params()))
    sim.set_solvent(pp)
    seeds = sim.next_seeds()
    sim.step(1)
    got = sim.get_solvent()
    ref = oracle.dpd_step(L, pp, systems.dpd_params(), seeds, 1.0, None, 5e-4)
    assert len(got) == len(pp)
    assert np.abs(got[:, :3] - ref[:, :3]).max() < 1e-6
    assert np.abs(got[:, 3:] - ref[:, 3:]).max() < 1e-3
    assert C.device_error() == 0
    sim.close()


def test_field_without_a_wall():
    """A field negative everywhere: nothing freezes, the wall has no
    particles, its forces and bounce-back change nothing."""
    import ctc_b200 as C
    L = (8, 8, 8)
    D = np.full((8, 8, 8), -3.0, np.float32)
    sdf = C.Sdf(L, grid=((8, 8, 8), (8.0, 8.0, 8.0), D))
    pp = systems.solvent(L, seed=5)
    w = C.Wall(sdf, pp)
    assert np.array_equal(w.bulk, pp)
    pos, st = w.particles()
    assert len(pos) == 0 and (st == 0).all()
    d = dev(pp)
    ff = torch.zeros((len(pp), 3), device="cuda")
    w.force(C.DpdParams(*systems.dpd_params()), d, ff)
    w.bounce(5e-4, d)
    assert ff.abs().max().item() == 0
    assert torch.equal(d, dev(pp))
    assert C.device_error() == 0


def test_membranes_without_cells():
    import ctc_b200 as C
    V, F = mesh.read_off(os.path.join(GOLDEN, "rbc.642.off"))
    A, Vol = mesh.area_volume(V, F)
    mod = C.RbcForce(F, len(V), 4)
    for mode in ("kantor", "juelicher"):
        mod.set_bending(mode)
        ff = torch.zeros((0, 3), device="cuda")
        mod.apply(C.RbcParams(**systems.rbc_params(A, Vol)), torch.zeros((0, 6), device="cuda"), ff)
    assert C.device_error() == 0
