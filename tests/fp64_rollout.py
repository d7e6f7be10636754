"""FP64 host reference of the differentiable solvent rollout (test helper).

The same discrete dynamics as the device rollout with stable keys, in double
precision on the host, for small periodic boxes: every pair within the cutoff
under the minimum image (the device's bulk + halo pair set when L >= 3), the
DPD pair force of src/pair/dev.h:111-139 with the random number of the pair
held fixed (its float value from the oracle's restatement of
src/math/rnd/dev.h, keyed by the two particle ids), then v += F/m dt,
x += v dt and the periodic wrap.  Gradients come from central differences in
double, which makes this an independent check of the hand-written adjoint.
"""
import numpy as np

import oracle


def _pairs(L, x):
    """All i < j with minimum-image distance^2 < 1: (i, j, dr) with dr = x_i - x_j."""
    n = len(x)
    iu, ju = np.triu_indices(n, 1)
    out_i, out_j, out_d = [], [], []
    step = 1 << 22
    for s in range(0, len(iu), step):
        i, j = iu[s:s + step], ju[s:s + step]
        d = x[i] - x[j]
        d -= L * np.round(d / L)
        r2 = (d * d).sum(1)
        m = r2 < 1.0
        out_i.append(i[m]); out_j.append(j[m]); out_d.append(d[m])
    return np.concatenate(out_i), np.concatenate(out_j), np.concatenate(out_d)


def forces(L, x, v, ids, theta, spow, kBT, dt, seed):
    a, g = theta
    s = np.sqrt(2.0 * kBT * g / dt)
    i, j, d = _pairs(L, x)
    r2 = (d * d).sum(1)
    keep = r2 >= 1e-6
    i, j, d, r2 = i[keep], j[keep], d[keep], r2[keep]
    r = np.sqrt(r2)
    e = d / r[:, None]
    dv = v[i] - v[j]
    ev = (e * dv).sum(1)
    w = np.maximum(1.0 - r, 0.0)
    wr = w ** spow
    gi, gj = ids[i].astype(np.uint32), ids[j].astype(np.uint32)
    rnd = oracle.mean0var1_batch(np.float32(seed), np.maximum(gi, gj), np.minimum(gi, gj), unsigned=True)
    phi = (-g * wr * ev + s * rnd.astype(np.float64)) * wr + a * w
    f = phi[:, None] * e
    F = np.zeros_like(x)
    np.add.at(F, i, f)
    np.add.at(F, j, -f)
    return F


def rollout(L, pp, theta, K, seeds, spow=0.25, kBT=0.0444, dt=5e-4, mass=1.0):
    """Final (x, v) [float64, by particle id] after K steps from pp (AoS)."""
    L = np.asarray(L, np.float64)
    lo = -np.floor(L / 2)
    x = pp[:, :3].astype(np.float64)
    v = pp[:, 3:].astype(np.float64)
    ids = np.arange(len(pp))
    for t in range(K):
        x = lo + np.mod(x - lo, L)               # the periodic wrap at the start of a step
        F = forces(L, x, v, ids, theta, spow, kBT, dt, seeds[t])
        v = v + F / mass * dt
        x = x + v * dt
    return x, v


def step_seeds(K):
    """The solvent seeds of K steps: the trunk seeded (0, 0, 0, 0), once a step."""
    k = oracle.Kiss(0, 0, 0, 0)
    return [k.get() for _ in range(K)]


def full_seeds(K):
    """Per step: the solvent seed (trunk (0, 0, 0, 0), once a step) and the
    FSI seed (trunk rnd_ini(1908, 1409, 290, 12968), the first of its two
    draws a step; with stable keys the bulk seed keys every FSI pair)."""
    kb, kf = oracle.Kiss(0, 0, 0, 0), oracle.Kiss(1908, 1409, 290, 12968)
    out = []
    for _ in range(K):
        s = kb.get()
        f = kf.get()
        kf.get()
        out.append((s, f))
    return out


def _rbc_wrap(L, pv, nv):
    """A cell whose bounding-box centre left [-L/2, L/2) re-enters whole."""
    lo = -(L // 2)
    for c in range(len(pv) // nv):
        q = pv[c * nv:(c + 1) * nv]
        r = 0.5 * (q[:, :3].min(0) + q[:, :3].max(0))
        d = -1 + (r >= lo).astype(int) + (r >= lo + L).astype(int)
        q[:, :3] -= d * L


def full_rollout(L, pp, pv, tri, nv, theta, rbc, fsi, K, seeds, spow=0.25, kBT=0.0444, dt=5e-4, mass=1.0,
                 mmass=0.5):
    """Solvent + membranes, K steps in double with stable keys, the step of
    the device rollout: wrap, solvent pairs (a, gamma = theta[:2], sigma from
    gamma), FSI, membrane forces (ks, kb = theta[2:]), then both updates.
    Returns the final solvent (AoS, by particle id) and vertices (AoS)."""
    Li = np.asarray(L, np.int64)
    Lf = Li.astype(np.float64)
    lo = -(Li // 2).astype(np.float64)
    x = np.array(pp, np.float64)
    xv = np.array(pv, np.float64)
    ids = np.arange(len(x), dtype=np.int32)
    a, g, ks, kb = (float(t) for t in theta)
    s = np.sqrt(2.0 * kBT * g / dt)
    par = dict(rbc, ks=ks, kb=kb)
    for t in range(K):
        x[:, :3] = lo + np.mod(x[:, :3] - lo, Lf)
        _rbc_wrap(Li, xv, nv)
        F, Fv = oracle.rollout_forces_f64(tuple(int(l) for l in Li), x, ids, (a, g, s, spow), seeds[t][0], xv, fsi,
                                          seeds[t][1], tri, nv, par)
        x[:, 3:] += F / mass * dt
        x[:, :3] += x[:, 3:] * dt
        xv[:, 3:] += Fv / mmass * dt
        xv[:, :3] += xv[:, 3:] * dt
    return x, xv
