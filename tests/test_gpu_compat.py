"""The drop-in boundary executed: one step of the path -- clist_build, the
bulk and halo solvent forces, fsi_bulk + fsi_halo, the body force, the
solvent update, rbc_force_apply with Kantor bending, the membrane update --
through the reference's own module signatures (ctc_b200/compat/udx_drive.cpp
linked with udx_compat.o, libctc_b200.so and the reference's mesh-reading,
parameter and utils modules built from their sources), against the same step
through the ctypes front end of the C ABI.  The halo and the FSI images come
in as the reference's exchange would deliver them (the solvent fragments
LFrag26 / RFrag26, the images Pap26 with their counts); the ctypes path
builds both on the device from the cell lists and the vertices.

Both draw their seeds from fresh modules' trunks, so the random forces are the
same.  Cell lists and the sorted order bit for bit; forces within 1e-5
relative (max-norm per particle: the float atomics of the two paths add in
different orders); positions after the step within 1e-6."""
import os
import struct
import subprocess

import numpy as np
import pytest

import oracle
from ctc_b200 import mesh, systems
from oracle import refkern

from .conftest import GOLDEN

torch = pytest.importorskip("torch")
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVE = os.path.join(ROOT, "ctc_b200", "compat", "_build", "udx_drive")
pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not os.path.exists(DRIVE), reason="udx_drive not built")]


def _rel_err(f, ref):
    f = np.asarray(f, np.float64).reshape(-1, 3)
    ref = np.asarray(ref, np.float64).reshape(-1, 3)
    mag = np.abs(ref).max(1)
    act = mag[mag > 0]
    floor = 0.1 * act.mean() if len(act) else 1.0
    return float((np.abs(f - ref).max(1) / np.maximum(mag, floor)).max())


def _system(L):
    off = os.path.join(GOLDEN, "rbc.642.off")
    V, F = mesh.read_off(off)
    nv = len(V)
    rng = np.random.default_rng(31)
    ps = systems.solvent(L, seed=32)
    pv = np.zeros((2 * nv, 6), np.float32)
    pv[:nv, :3] = V @ mesh.random_rotation(rng).T + np.array([L[0] / 2 - 2.0, 0.0, 0.0])   # across +x
    pv[nv:, :3] = V @ mesh.random_rotation(rng).T + np.array([-1.0, -2.0, 1.0])
    pv[:, 3:] = rng.normal(0, 0.3, (2 * nv, 3))
    A, Vol = mesh.area_volume(V, F)
    par = systems.rbc_params(A * 1.02, Vol * 0.98)
    return off, ps, pv, F, nv, par


def _write_input(path, L, ps, dpd, kBT, dt, bodyf, off, pv, nc, par, fsi, frags, images):
    with open(path, "wb") as f:
        f.write(struct.pack("<3i", *L))
        f.write(struct.pack("<i", len(ps)))
        f.write(np.ascontiguousarray(ps, "<f4").tobytes())
        f.write(struct.pack("<5f", dpd[0], dpd[1], dpd[3], kBT, dt))
        f.write(struct.pack("<3f", *bodyf))
        b = off.encode()
        f.write(struct.pack("<i", len(b)) + b)
        f.write(struct.pack("<i", nc))
        f.write(np.ascontiguousarray(pv, "<f4").tobytes())
        f.write(np.array([par[k] for k in refkern._RBC_FIELDS], "<f4").tobytes())
        f.write(struct.pack("<2f", fsi[0], fsi[1]))
        for ii, fss in frags:
            f.write(struct.pack("<i", len(ii)) + np.asarray(ii, "<i4").tobytes())
            f.write(struct.pack("<i", len(fss) - 1) + np.asarray(fss, "<i4").tobytes())
        counts, vert, img = images
        f.write(np.asarray(counts, "<i4").tobytes())
        f.write(struct.pack("<i", len(vert)) + np.asarray(vert, "<i4").tobytes())
        f.write(np.ascontiguousarray(img, "<f4").tobytes())


def _read_output(path):
    d = open(path, "rb").read()
    o = 0
    n = struct.unpack_from("<i", d, o)[0]; o += 4
    pp = np.frombuffer(d, "<f4", 6 * n, o).reshape(n, 6); o += 24 * n
    ff = np.frombuffer(d, "<f4", 3 * n, o).reshape(n, 3); o += 12 * n
    nvt = struct.unpack_from("<i", d, o)[0]; o += 4
    fv = np.frombuffer(d, "<f4", 3 * nvt, o).reshape(nvt, 3); o += 12 * nvt
    pv = np.frombuffer(d, "<f4", 6 * nvt, o).reshape(nvt, 6)
    return pp, ff, fv, pv


@pytest.mark.parametrize("L", [(12, 12, 12), (16, 12, 10)])
def test_step_through_reference_signatures_equals_ctypes_path(L, tmp_path):
    import ctc_b200 as C
    off, ps, pv, F, nv, par = _system(L)
    dpd = systems.dpd_params()
    fsi = (0.0, 8.0, dpd[2], 0.25)
    kBT, dt, bodyf = systems.KBT, systems.DT, (0.01, 0.0, 0.0)
    counts, starts, order, ps_sorted = oracle.clist_build(L, ps)
    frags = refkern.fragments(L, starts, counts)
    images = refkern.images(L, pv)
    assert len(images[1]) > 0
    inp, out = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    _write_input(inp, L, ps, dpd, kBT, dt, bodyf, off, pv, 2, par, fsi, frags, images)
    r = subprocess.run([DRIVE, inp, out], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    gp, gff, gfv, gpv = _read_output(out)

    # the same step through the ctypes front end
    n, nvt = len(ps), len(pv)
    P, starts_d, counts_d, ids = C.Clist(L, n).build(torch.as_tensor(ps, device="cuda"))
    assert np.array_equal(starts_d.cpu().numpy(), starts) and np.array_equal(ids.cpu().numpy(), order)
    D = C.DpdParams(*dpd)
    ff = torch.zeros((n, 3), device="cuda")
    mod = C.FluForces(L, n)
    mod.bulk_apply(D, P, starts_d, counts_d, ff)
    mod.halo_apply(D, P, starts_d, counts_d, ff)
    V = torch.as_tensor(pv, device="cuda")
    fv = torch.zeros((nvt, 3), device="cuda")
    C.Fsi(L, nvt, n).apply(C.DpdParams(*fsi), V, P, starts_d, counts_d, fv, ff)
    C.bforce_apply_cste(1.0, bodyf, ff)
    C.bforce_apply_cste(systems.RBC_MASS, bodyf, fv)
    ff_h = ff.cpu().numpy()
    C.scheme_move_apply(dt, 1.0, ff, P)
    C.RbcForce(F, nv, 2).apply(C.RbcParams(**par), V, fv)
    fv_h = fv.cpu().numpy()
    C.scheme_move_apply(dt, systems.RBC_MASS, fv, V)
    torch.cuda.synchronize()
    assert C.device_error() == 0

    assert _rel_err(gff, ff_h) < 1e-5
    assert _rel_err(gfv, fv_h) < 1e-5
    assert np.abs(gp[:, :3] - P.cpu().numpy()[:, :3]).max() < 1e-6
    assert np.abs(gpv[:, :3] - V.cpu().numpy()[:, :3]).max() < 1e-6
