"""Walls on the device (src/wall): the field evaluation, labels, frozen wall,
wall forces, bounce-back and repulsion of this build against the reference's
own wall kernels compiled from its sources (oracle/_ref/librefkern.so, with
the field on a real 3D texture as the reference binds it) and against the
oracle.

Bars: the field and labels bit for bit against the reference's kernels; the
forces per particle within 1e-5 of the particle's force (floored at 0.1 x
the mean): the reference adds its three partial sums atomically in an
unspecified order; bounce-back positions and velocities within 1e-5.  Against
the CPU oracle: forces within 2e-3 as for the other pair forces (the device's
rsqrtf/powf are the reference's fast-math instructions, the oracle's the
correctly rounded libm ones), bounced positions and velocities within 1e-3
(two Newton steps on field values that differ in the last bits)."""
import os

import numpy as np
import pytest

import oracle
from oracle import refkern
from ctc_b200 import systems

from .conftest import GOLDEN

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refkern.available(), reason="oracle/_ref/librefkern.so not built")]

SDF = os.path.join(GOLDEN, "sdf")


def dev(x):
    return torch.as_tensor(np.ascontiguousarray(x), device="cuda")


def rel_err(f, ref):
    f = np.asarray(f, np.float64).reshape(-1, 3)
    ref = np.asarray(ref, np.float64).reshape(-1, 3)
    mag = np.abs(ref).max(1)
    return float((np.abs(f - ref).max(1) / np.maximum(mag, 0.1 * mag.mean())).max())


def _setup(name, L):
    import ctc_b200 as C
    path = os.path.join(SDF, name)
    sdf = C.Sdf(L, path=path)
    T, tex, o, s, thr = sdf.texture()
    ref = refkern.RefSdf(tex, o, s, thr)
    q = oracle.Sdf(*oracle.sdf_read(path), L)
    assert np.array_equal(tex.reshape(-1), q.tex)
    return C, sdf, ref, q


def _solvent(L, seed, margin_away=True, q=None):
    pp = systems.solvent(L, seed=seed)
    if margin_away and q is not None:   # no particle within 1e-4 of a label boundary
        s = q.eval(pp)
        pp = pp[(np.abs(s) > 1e-4) & (np.abs(s - 2) > 1e-4)]
    return pp


def _wvels(C):
    return [(C.wvel("cste", u=(0.5, -0.2, 0.1)), oracle.Wvel(0, (0.5, -0.2, 0.1), 0, 0, 0, 0, 0)),
            (C.wvel("shear", gdot=5.0, vdir=0, gdir=2), oracle.Wvel(1, (0, 0, 0), 5.0, 0, 2, 0, 0))]


@pytest.mark.parametrize("name,L", [("wall.dat", (16, 16, 16)), ("yplates.dat", (16, 12, 20))])
def test_field_and_labels_bitwise(name, L):
    C, sdf, ref, q = _setup(name, L)
    rng = np.random.default_rng(1)
    pp = np.zeros((200000, 6), np.float32)
    pp[:, :3] = rng.uniform(-0.5, 0.5, (len(pp), 3)) * (np.array(L) + 10)   # the box and most of the margin
    d = dev(pp)
    a, b = torch.zeros(len(pp), device="cuda"), torch.zeros(len(pp), device="cuda")
    sdf.eval(d, a)
    ref.eval(d, b)
    assert torch.equal(a, b)
    assert np.abs(a.cpu().numpy() - q.eval(pp)).max() < 1e-5
    la = torch.zeros(len(pp), dtype=torch.int32, device="cuda")
    lb = torch.zeros_like(la)
    sdf.label(d, la)
    ref.label(d, lb)
    assert torch.equal(la, lb)
    ref.close()


def test_freeze_vs_oracle():
    C, sdf, ref, q = _setup("wall.dat", (16, 16, 16))
    L = (16, 16, 16)
    pp = _solvent(L, 3, q=q)
    w = C.Wall(sdf, pp)
    bulk, wpos, ws = q.freeze(pp)
    assert np.array_equal(w.bulk, bulk)
    pos, st = w.particles()
    assert np.array_equal(st, ws) and np.array_equal(pos, wpos)
    assert len(bulk) < len(pp) and len(pos) > 0
    ref.close()


@pytest.mark.parametrize("name,L", [("wall.dat", (16, 16, 16)), ("yplates.dat", (16, 12, 20))])
def test_wall_force_vs_reference_kernel(name, L):
    C, sdf, ref, q = _setup(name, L)
    pp = _solvent(L, 5, q=q)
    w = C.Wall(sdf, pp)
    bulk = w.bulk.copy()
    bulk[:, 3:] = np.random.default_rng(6).normal(0, 0.3, (len(bulk), 3))
    pos, st = w.particles()
    dpd = systems.dpd_params()
    for wv, owv in _wvels(C):
        w.set_vel(wv)
        ff = torch.zeros((len(bulk), 3), device="cuda")
        w.force(C.DpdParams(*dpd), dev(bulk), ff, seed=0.37)
        fr = torch.zeros_like(ff)
        rw = refkern.RefWvel(owv.type, owv.u, owv.gdot, owv.vdir, owv.gdir, owv.half, owv.h)
        ref.force(L, dev(pos), dev(st), rw, dpd, 0.37, dev(bulk), fr)
        f, r = ff.cpu().numpy(), fr.cpu().numpy()
        near = np.abs(r).sum(1) > 0
        assert near.sum() > 100 and (np.abs(f[~near]) == 0).all()
        assert rel_err(f[near], r[near]) < 1e-5
        o = q.force(pos, st, owv, dpd, 0.37, bulk)
        assert rel_err(f[near], o[near]) < 2e-3
    assert C.device_error() == 0
    ref.close()


def test_wall_force_draws_the_tickets_seeds():
    C, sdf, ref, q = _setup("wall.dat", (16, 16, 16))
    L = (16, 16, 16)
    pp = _solvent(L, 7, q=q)
    w = C.Wall(sdf, pp)
    pos, st = w.particles()
    dpd = systems.dpd_params()
    k = oracle.Kiss(42, 42, 42, 42)
    bulk = w.bulk
    for _ in range(2):
        ff = torch.zeros((len(bulk), 3), device="cuda")
        w.force(C.DpdParams(*dpd), dev(bulk), ff)
        o = q.force(pos, st, oracle.Wvel(0, (0, 0, 0), 0, 0, 0, 0, 0), dpd, k.get(), bulk)
        f = ff.cpu().numpy()
        near = np.abs(o).sum(1) > 0
        assert rel_err(f[near], o[near]) < 2e-3
    ref.close()


@pytest.mark.parametrize("name,L", [("wall.dat", (16, 16, 16)), ("yplates.dat", (16, 12, 20))])
def test_bounce_vs_reference_kernel(name, L):
    """Bulk particles pushed into the wall by v dt bounce back: this build
    against the reference's kernel and the oracle."""
    C, sdf, ref, q = _setup(name, L)
    pp = _solvent(L, 9, q=q)
    w = C.Wall(sdf, pp)
    bulk = w.bulk.copy()
    rng = np.random.default_rng(10)
    dt = 0.05
    bulk[:, 3:] = rng.normal(0, 3.0, (len(bulk), 3))
    moved = bulk.copy()
    moved[:, :3] += dt * bulk[:, 3:]
    inside = q.eval(moved) >= 0
    assert inside.sum() > 50
    for wv, owv in _wvels(C):
        w.set_vel(wv)
        a = dev(moved)
        w.bounce(dt, a)
        b = dev(moved)
        ref.bounce(L, refkern.RefWvel(owv.type, owv.u, owv.gdot, owv.vdir, owv.gdir, owv.half, owv.h), dt, b)
        a, b = a.cpu().numpy(), b.cpu().numpy()
        assert np.array_equal(a[~inside], moved[~inside])
        assert np.abs(a - b).max() < 1e-5
        o = q.bounce(owv, dt, moved)
        assert np.abs(a - o).max() < 1e-3      # Newton steps on the oracle's unfused field values
        assert (q.eval(a[inside]) < 0).mean() > 0.99      # back in the bulk
    ref.close()


def test_repulse_vs_reference_kernel():
    C, sdf, ref, q = _setup("wall.dat", (16, 16, 16))
    rng = np.random.default_rng(11)
    pp = np.zeros((50000, 6), np.float32)
    pp[:, :3] = rng.uniform(-8, 8, (len(pp), 3))
    w = C.Wall(sdf, np.zeros((0, 6), np.float32))
    a = torch.zeros((len(pp), 3), device="cuda")
    b = torch.zeros_like(a)
    w.repulse(2.0, dev(pp), a)
    ref.repulse(2.0, dev(pp), b)
    a, b = a.cpu().numpy(), b.cpu().numpy()
    near = np.abs(b).sum(1) > 0
    assert near.sum() > 100
    assert rel_err(a[near], b[near]) < 1e-5
    assert rel_err(a[near], q.repulse(2.0, pp)[near]) < 2e-3
    ref.close()


def _wall_step(L, q, wpos, ws, owv, ps, dpd, seeds, wseed, bodyf, dt):
    """One solvent step with walls in the reference's order (src/sim/imp/
    run.h:8-68 with forces_wall after the DPD forces, bounce_wall after the
    update)."""
    counts, starts, ps = oracle.distribute(L, ps)
    fs = oracle.dpd_bulk(L, ps, starts, dpd, seeds[0]) + oracle.dpd_halo(L, ps, starts, counts, dpd, seeds[1:])
    fs = fs + q.force(wpos, ws, owv, dpd, wseed, ps)
    fs = oracle.body_force(fs, 1.0, np.asarray(bodyf, np.float32))
    ps = oracle.move(ps, fs, dt, 1.0)
    out = q.bounce(owv, dt, ps)
    return out, (out != ps).any(1)


@pytest.mark.parametrize("kind", ["cste", "shear"])
def test_sim_step_with_walls_vs_oracle(kind):
    import ctc_b200 as C
    L = (16, 16, 16)
    path = os.path.join(SDF, "wall.dat")
    q = oracle.Sdf(*oracle.sdf_read(path), L)
    ps0 = _solvent(L, 13, q=q)
    dpd = systems.dpd_params()
    bodyf = (0.0333333, 0.0, 0.0)
    sdf = C.Sdf(L, path=path)
    sim = C.Sim(L, len(ps0), C.DpdParams(*dpd), mass=1.0, dt=systems.DT, bodyf=bodyf)
    sim.set_solvent(ps0)
    sim.step(1)
    if kind == "cste":
        wv, owv = C.wvel("cste"), oracle.Wvel(0, (0, 0, 0), 0, 0, 0, 0, 0)
    else:
        wv, owv = C.wvel("shear", gdot=5.0, vdir=0, gdir=2), oracle.Wvel(1, (0, 0, 0), 5.0, 0, 2, 0, 0)
    before = sim.get_solvent()
    k0 = oracle.Kiss(0, 0, 0, 0)
    kh = [oracle.Kiss.halo(f) for f in range(26)]
    for _ in range(1):                   # the trunks' draws of the first step
        k0.get()
        [k.get() for k in kh]
    sim.set_walls(sdf, wv)
    bulk, wpos, ws = q.freeze(before)
    rs = sim.get_solvent()
    assert np.array_equal(rs, bulk)
    kw = oracle.Kiss(42, 42, 42, 42)
    for step in range(3):
        seeds = np.array([k0.get()] + [k.get() for k in kh], np.float32)
        sim.step(1)
        rs, bounced = _wall_step(L, q, wpos, ws, owv, rs, dpd, seeds, kw.get(), bodyf, systems.DT)
        gs = sim.get_solvent()
        assert len(gs) == len(rs)
        # particles that bounced: the bar of the bounce test against the oracle
        assert np.abs(gs[~bounced, :3] - rs[~bounced, :3]).max() < 2e-6
        assert np.abs(gs[:, 3:] - rs[:, 3:]).max() < 1e-3
        assert np.abs(gs[bounced] - rs[bounced]).max(initial=0) < 1e-3
        rs = gs
    assert C.device_error() == 0
    sim.close()


def test_sim_walls_channel_flow_and_graph_replay():
    """Poiseuille flow between the plates of wall.dat: no particle crosses
    into the wall, the body force drives a flow, and graph replay follows the
    direct launches."""
    import ctc_b200 as C
    L = (16, 16, 16)
    path = os.path.join(SDF, "wall.dat")
    q = oracle.Sdf(*oracle.sdf_read(path), L)
    sdf = C.Sdf(L, path=path)
    dpd = systems.dpd_params()
    out = []
    for graph in (False, True):
        sim = C.Sim(L, 10 * 16 ** 3, C.DpdParams(*dpd), mass=1.0, dt=systems.DT, bodyf=(0.5, 0.0, 0.0),
                    rng=C.CTC_RNG_STABLE)
        sim.set_solvent(systems.solvent(L, seed=17))
        sim.set_walls(sdf, C.wvel("cste"))
        sim.set_graph(graph)
        sim.step(200)
        gs = sim.get_solvent()
        assert (q.eval(gs) < 0).all()
        assert gs[:, 3].mean() > 0.02
        out.append(gs)
        sim.close()
    assert np.abs(out[0] - out[1]).max() < 1e-3
    assert C.device_error() == 0


def test_wall_restart_template(tmp_path):
    """wall_strt_dump_templ then a wall from the template: the same wall, and
    a system restarted with it steps as the original."""
    import ctc_b200 as C
    L = (16, 16, 16)
    path = os.path.join(SDF, "wall.dat")
    q = oracle.Sdf(*oracle.sdf_read(path), L)
    sdf = C.Sdf(L, path=path)
    pp = _solvent(L, 19, q=q)
    w = C.Wall(sdf, pp)
    w.strt_dump_templ(tmp_path)
    t = C.restart_read_pp(tmp_path, "wall.pp", "templ")
    pos, st = w.particles()
    assert np.array_equal(t[:, :3], pos[:, :3]) and (t[:, 3:] == 0).all()
    w2 = C.Wall.strt(sdf, tmp_path)
    pos2, st2 = w2.particles()
    assert np.array_equal(pos, pos2) and np.array_equal(st, st2)
    # a wall from the particles themselves, in another order: the same cell list
    w3 = C.Wall.from_particles(sdf, pos[::-1])
    pos3, st3 = w3.particles()
    assert np.array_equal(st, st3)
    rows = lambda a: a[np.lexsort(a.T[::-1])]
    assert np.array_equal(rows(pos3), rows(pos))
    dpd = systems.dpd_params()
    a = C.Sim(L, len(pp), C.DpdParams(*dpd), mass=1.0, dt=systems.DT, bodyf=(0.1, 0.0, 0.0))
    a.set_solvent(pp)
    a.set_walls(sdf, C.wvel("cste"))
    a.wall_strt_dump_templ(tmp_path / "sim")
    b = C.Sim(L, len(pp), C.DpdParams(*dpd), mass=1.0, dt=systems.DT, bodyf=(0.1, 0.0, 0.0))
    b.set_solvent(a.get_solvent())
    b.set_walls_strt(sdf, tmp_path / "sim", C.wvel("cste"))
    a.step(2)
    b.step(2)
    assert np.abs(a.get_solvent() - b.get_solvent()).max() < 1e-5
    a.close()
    b.close()
    assert C.device_error() == 0


def test_sim_walls_with_membranes():
    """A cell in the channel between the plates: the wall forces (FSI
    parameters) and the repulsion act on its vertices (the module's forces
    on the same state), the membranes set after the walls are covered, and
    after some steps no vertex is inside the wall."""
    import ctc_b200 as C
    from ctc_b200 import mesh
    L = (16, 16, 16)
    path = os.path.join(SDF, "wall.dat")
    q = oracle.Sdf(*oracle.sdf_read(path), L)
    sdf = C.Sdf(L, path=path)
    X, F = mesh.rbc_template()
    pv = np.zeros((len(X), 6), np.float32)
    pv[:, :3] = X
    pv[:, 2] += 4.2                        # its top within the plate's reach
    s = q.eval(pv)
    assert (s < -0.5).all() and (s > -1.4).sum() > 10
    A, V = mesh.area_volume(X, F)
    par = systems.rbc_params(A, V)
    dpd = systems.dpd_params()
    fsi = C.DpdParams(0.0, 8.0, dpd[2], 0.25)
    sim = C.Sim(L, 10 * 16 ** 3, C.DpdParams(*dpd), mass=1.0, dt=systems.DT)
    sim.set_solvent(_solvent(L, 23, q=q))
    sim.set_walls(sdf, C.wvel("cste"), lam=4.0)
    sim.set_membranes(pv, F, len(X), par, fsi, mass=systems.RBC_MASS)
    # the module's forces on these vertices: some near the plate feel it
    w = C.Wall(sdf, np.zeros((0, 6), np.float32))
    fw = torch.zeros((len(pv), 3), device="cuda")
    w.repulse(4.0, dev(pv), fw)
    assert (fw.abs().sum(1) > 0).sum().item() > 10
    sim.step(20)
    gv = sim.get_membranes()
    assert np.isfinite(gv).all()
    assert (q.eval(gv) < 0).all()
    assert C.device_error() == 0
    sim.close()


def test_cells_in_the_wall_are_removed():
    """objects_remove_from_wall: of two cells, the one that crosses a plate
    leaves when the walls are set; sdf_who_stays names the other."""
    import ctc_b200 as C
    from ctc_b200 import mesh
    L = (16, 16, 16)
    path = os.path.join(SDF, "wall.dat")
    q = oracle.Sdf(*oracle.sdf_read(path), L)
    sdf = C.Sdf(L, path=path)
    X, F = mesh.rbc_template()
    nv = len(X)
    pv = np.zeros((2 * nv, 6), np.float32)
    pv[:nv, :3] = X
    pv[nv:, :3] = X
    pv[nv:, 2] += 6.5                     # through the upper plate
    s = q.eval(pv)
    assert (s[:nv] < 0).all() and (s[nv:] >= 0).any()
    assert list(sdf.who_stays(dev(pv), nv)) == [0]
    A, V = mesh.area_volume(X, F)
    dpd = systems.dpd_params()
    sim = C.Sim(L, 10 * 16 ** 3, C.DpdParams(*dpd), mass=1.0, dt=systems.DT)
    sim.set_solvent(_solvent(L, 29, q=q))
    sim.set_membranes(pv, F, nv, systems.rbc_params(A, V), C.DpdParams(0.0, 8.0, dpd[2], 0.25),
                      mass=systems.RBC_MASS)
    sim.set_walls(sdf, C.wvel("cste"))
    assert sim.mnc == 1
    gv = sim.get_membranes()
    assert np.array_equal(gv, pv[:nv])
    sim.step(3)
    assert C.device_error() == 0
    sim.close()


def test_sim_everything_together_graph_and_direct():
    """Walls, membranes with contact, the membrane random force and
    Juelicher bending in one step: graph replay follows the direct
    launches, nothing enters the wall, no kernel records a failure."""
    import ctc_b200 as C
    from ctc_b200 import mesh
    L = (16, 16, 16)
    path = os.path.join(SDF, "wall.dat")
    q = oracle.Sdf(*oracle.sdf_read(path), L)
    sdf = C.Sdf(L, path=path)
    X, F = mesh.rbc_template()
    nv = len(X)
    pv = np.zeros((2 * nv, 6), np.float32)
    pv[:nv, :3] = X + (-3.0, 0.0, -1.5)
    pv[nv:, :3] = X + (3.0, 0.0, 1.5)
    A, V = mesh.area_volume(X, F)
    dpd = systems.dpd_params()
    ps = _solvent(L, 31, q=q)
    out = []
    for graph in (False, True):
        sim = C.Sim(L, len(ps), C.DpdParams(*dpd), mass=1.0, dt=systems.DT, bodyf=(0.2, 0.0, 0.0),
                    rng=C.CTC_RNG_STABLE)
        sim.set_solvent(ps)
        sim.set_membranes(pv, F, nv, systems.rbc_params(A, V), C.DpdParams(0.0, 8.0, dpd[2], 0.25),
                          mass=systems.RBC_MASS)
        sim.set_walls(sdf, C.wvel("shear", gdot=1.0, vdir=0, gdir=2), lam=2.0)
        sim.set_contact(C.DpdLjParams(dpd[0], dpd[1], dpd[2], 0.25, 0.3, 0.44))
        sim.set_membrane_noise(True, seed=5)
        sim.set_bending("juelicher")
        sim.set_graph(graph)
        sim.step(20)
        gs, gv = sim.get_solvent(), sim.get_membranes()
        assert np.isfinite(gs).all() and np.isfinite(gv).all()
        assert (q.eval(gs) < 0).all() and (q.eval(gv) < 0).all()
        out.append((gs, gv))
        sim.close()
    assert np.abs(out[0][0] - out[1][0]).max() < 1e-3
    assert np.abs(out[0][1] - out[1][1]).max() < 1e-3
    assert C.device_error() == 0
