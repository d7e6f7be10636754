"""Seeded synthetic systems of the benchmark configurations.

There is no public dataset for this path; every input is generated here from
a seed: uniform solvent at number density rho in a periodic box of L unit
cells ([-L/2, L/2) per axis, lower corner -(L//2)), velocities Gaussian with
variance kBT/m per component.
"""
import numpy as np

# DPD parameters shared by the configurations (rc = 1)
A_DPD, GAMMA, SPOW, KBT, DT = 2.5, 8.0, 0.25, 0.0444, 5e-4


def box_lo(L):
    return np.array([-(int(x) // 2) for x in L], np.float64)


def solvent(L, rho=10, kBT=KBT, mass=1.0, seed=1, n=None):
    """(n, 6) float32 AoS particles, uniform in the box, Maxwellian velocities."""
    rng = np.random.default_rng(seed)
    L = np.asarray(L, np.int64)
    if n is None:
        n = int(rho * L.prod())
    lo = box_lo(L)
    r = lo + rng.random((n, 3)) * L
    r = r.astype(np.float32)
    hi = (lo + L).astype(np.float32)
    r = np.minimum(r, np.nextafter(hi, np.float32(-np.inf)))   # stay inside after rounding
    v = rng.normal(0.0, np.sqrt(kBT / mass), (n, 3)).astype(np.float32)
    pp = np.empty((n, 6), np.float32)
    pp[:, :3] = r
    pp[:, 3:] = v
    return pp


def dpd_params(a=A_DPD, g=GAMMA, kBT=KBT, dt=DT, spow=SPOW):
    """(a, g, s, spow) with s = sqrt(2 kBT g / dt) in double, stored as float
    (src/pair/imp/main.h:54-62)."""
    s = float(np.float32(np.sqrt(2.0 * kBT * g / dt)))
    return (float(np.float32(a)), float(np.float32(g)), s, float(np.float32(spow)))


# ---------------------------------------------------------------------------
# red blood cells
# ---------------------------------------------------------------------------
RBC_MASS = 0.5   # conf/default.cfg:49


def rbc_params(totArea, totVolume, kBT=KBT, ks=14.8):
    """Membrane parameters of the RBC configurations: WLC + POW x0 = 0.457,
    mpow = 2, kb = 40 kBT, ka = 4900, kv = 5000, kd = 200, phi = 0,
    gammaC = 10, gammaT = 0 (conf/rbc.lina.cfg with the configuration's kb, ka,
    kv), ks = 14.8 (conf/rbc.test.cfg; the configurations give no ks)."""
    return dict(gammaC=10.0, gammaT=0.0, kBT=kBT, kb=40.0 * kBT, phi=0.0, ks=ks, x0=0.457, mpow=2.0,
                ka=4900.0, kd=200.0, kv=5000.0, totArea=float(totArea), totVolume=float(totVolume))


def place_cells(L, nc, X, rng, margin=0.5):
    """nc copies of template X at random non-overlapping centres (bounding
    spheres of radius max|X| + margin, periodic distance) with uniform random
    rotations.  Returns (nc * nv, 3) float32 positions (cells not wrapped)."""
    from . import mesh
    L = np.asarray(L, np.float64)
    lo = box_lo(L)
    R = float(np.linalg.norm(X, axis=1).max()) + margin
    centres = []
    tries = 0
    while len(centres) < nc:
        tries += 1
        if tries > 200000:
            raise RuntimeError("cannot place %d cells in box %s" % (nc, L))
        c = lo + rng.random(3) * L
        ok = True
        for d in centres:
            dd = c - d
            dd -= L * np.round(dd / L)
            if np.dot(dd, dd) < (2 * R) ** 2:
                ok = False
                break
        if ok:
            centres.append(c)
    out = []
    for c in centres:
        Q = mesh.random_rotation(rng)
        out.append(X @ Q.T + c)
    return np.concatenate(out).astype(np.float32) if out else np.zeros((0, 3), np.float32)


def rbc_system(L, nc, seed=3, kBT=KBT, D=7.82):
    """Membrane vertices (nc * 642, 6) AoS with Maxwellian velocities (mass
    0.5), the triangle template and its parameters."""
    from . import mesh
    rng = np.random.default_rng(seed)
    X, F = mesh.rbc_template(D)
    r = place_cells(L, nc, X.astype(np.float64), rng)
    pv = np.zeros((len(r), 6), np.float32)
    pv[:, :3] = r
    pv[:, 3:] = rng.normal(0.0, np.sqrt(kBT / RBC_MASS), (len(r), 3))
    A, V = mesh.area_volume(X, F)
    return pv, F, rbc_params(A, V, kBT)


def batch_system(nbox=512, emin=8, emax=24, rbc_every=4, seed=5, rho=10):
    """The batched-boxes workload: nbox cubic periodic boxes with edges drawn
    uniformly from emin..emax, solvent at density rho, one RBC in every
    rbc_every-th box (index 0, rbc_every, ...).  Boxes with an edge below the
    cell diameter + 2 rc let an RBC interact with its own periodic image
    through FSI; its internal forces use unwrapped coordinates, so this is
    allowed.  Returns (L[nbox, 3], n[nbox], solvent AoS box after box,
    cells[nbox], membrane vertices AoS box after box, triangles, params)."""
    rng = np.random.default_rng(seed)
    edges = rng.integers(emin, emax + 1, size=nbox)
    L = np.stack([edges] * 3, axis=1).astype(np.int32)
    parts, n = [], []
    for k in range(nbox):
        pp = solvent(tuple(L[k]), rho=rho, seed=int(rng.integers(1 << 31)))
        parts.append(pp)
        n.append(len(pp))
    cells = np.array([1 if (rbc_every and k % rbc_every == 0) else 0 for k in range(nbox)], np.int32)
    pv, tri, par = [], None, None
    for k in range(nbox):
        if cells[k]:
            v, tri, par = rbc_system(tuple(L[k]), 1, seed=int(rng.integers(1 << 31)))
            pv.append(v)
    pv = np.concatenate(pv) if pv else np.zeros((0, 6), np.float32)
    if tri is None:
        from . import mesh
        X, tri = mesh.rbc_template(7.82)
        A, V = mesh.area_volume(X, tri)
        par = rbc_params(A, V)
    return L, np.array(n, np.int32), np.concatenate(parts), cells, pv, tri, par
