"""The differentiable rollout: the hand-written adjoint against central finite
differences of the device's own FP32 forward (step 1e-3) and against an FP64
host reference gradient, the checkpoint interval, and the autograd wrapper.

Losses are linear functionals sum(c . v) of the final velocities with fixed
random c, which depend strongly on every input; the configuration's loss
(mean vertex x-velocity) is exercised through the autograd wrapper."""
import numpy as np
import pytest

from ctc_b200 import systems

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _solvent_rollout(L=(6, 6, 6), seed=21):
    from ctc_b200.adjoint import Rollout
    pp = systems.solvent(L, seed=seed)
    r = Rollout(L, pp, systems.dpd_params(), systems.KBT, systems.DT)
    return r, pp


def _loss_cv(r, cv, cvv=None):
    pp, pv = r.final_state()
    l = float(np.dot(cv.ravel().astype(np.float64), pp[:, 3:].ravel().astype(np.float64)))
    if cvv is not None:
        l += float(np.dot(cvv.ravel().astype(np.float64), pv[:, 3:].ravel().astype(np.float64)))
    return l


def test_solvent_gradient_vs_fp64_reference():
    """d/da, d/dgamma and d/dx0 of sum(c . v_K) against central differences of
    an FP64 host rollout of the same dynamics (K = 4)."""
    from tests import fp64_rollout as R
    K = 4
    r, pp = _solvent_rollout()
    L = np.array((6, 6, 6), np.float64)
    theta = np.array([systems.A_DPD, systems.GAMMA, 0.0, 0.0])
    r.set_params(theta)
    rng = np.random.default_rng(5)
    cv = rng.normal(size=(len(pp), 3)).astype(np.float32)
    r.forward(K, 2)
    g = r.backward(cot=(None, cv, None, None))
    seeds = R.step_seeds(K)

    def f64(th, pp_):
        _, v = R.rollout(L, pp_, th, K, seeds)
        return float((cv.astype(np.float64) * v).sum())

    h = 1e-6
    for k in range(2):
        tp, tm = theta[:2].copy(), theta[:2].copy()
        tp[k] += h
        tm[k] -= h
        ref = (f64(tp, pp) - f64(tm, pp)) / (2 * h)
        assert abs(g["theta"][k] - ref) <= 1e-3 * abs(ref) + 1e-6, (k, g["theta"][k], ref)
    for (i, c) in [(0, 0), (7, 1), (100, 2)]:
        pp_p, pp_m = pp.astype(np.float64), pp.astype(np.float64)
        pp_p[i, c] += h
        pp_m[i, c] -= h
        ref = (f64(theta[:2], pp_p) - f64(theta[:2], pp_m)) / (2 * h)
        scale = np.abs(g["gx"]).max()
        assert abs(g["gx"][i, c] - ref) <= 1e-3 * scale, (i, c, g["gx"][i, c], ref, scale)
    r.close()


def _rbc_rollout(L=(16, 16, 16), seed=31, spow=None):
    from ctc_b200.adjoint import Rollout
    pp = systems.solvent(L, seed=seed)
    pv, tri, par = systems.rbc_system(L, 1, seed=seed + 1)
    dpd = list(systems.dpd_params())
    if spow is not None:
        dpd[3] = spow
    fsi = (0.0, 8.0, dpd[2], dpd[3])
    r = Rollout(L, pp, dpd, systems.KBT, systems.DT, pv=pv, tri=tri, rbc=par, fsi=fsi, mmass=systems.RBC_MASS)
    theta = np.array([systems.A_DPD, systems.GAMMA, par["ks"], par["kb"]])
    return r, pp, pv, theta


def test_full_system_gradient_vs_finite_differences():
    """Solvent + one red blood cell, K = 4 with checkpoints every 2 steps:
    d/d(a, gamma, ks, kb) of sum(c . v_K) over solvent and vertices against
    central differences of the device's FP32 forward (relative step 1e-2),
    to 2e-3 relative (1e-2 for kb).

    The dissipative weight here is (1 - r)^1: with the configurations'
    (1 - r)^0.25 the pair force has an unbounded slope at the cutoff, and the
    pairs within rounding of it carry derivative that no FP32 finite
    difference resolves (about 1 % of d/da, d/dgamma at this size; the FP64
    reference test above resolves them).  The kernels take spow as a
    parameter, so this checks the same code."""
    K, kck = 4, 2
    r, pp, pv, theta = _rbc_rollout(L=(12, 12, 12), spow=1.0)
    rng = np.random.default_rng(6)
    cv = rng.normal(size=(len(pp), 3)).astype(np.float32)
    cvv = rng.normal(size=(len(pv), 3)).astype(np.float32)
    r.set_params(theta)
    r.forward(K, kck)
    g = r.backward(cot=(None, cv, None, cvv))
    h = 1e-2
    for k in range(4):
        vals = []
        step = h * max(1.0, abs(theta[k]))
        for sgn in (1, -1):
            t = theta.copy()
            t[k] += sgn * step
            r.set_params(t)
            r.forward(K, kck)
            vals.append(_loss_cv(r, cv, cvv))
        fd = (vals[0] - vals[1]) / (2 * step)
        # kb: the bending share of this loss is small, and the FP32 finite
        # differences of it scatter by ~0.5 % between step sizes (the kinks of
        # pairs crossing the cutoff); with K = 1, where the loss is linear in
        # kb, the adjoint matches the secant to 2e-4
        tol = 1e-2 if k == 3 else 2e-3
        assert abs(g["theta"][k] - fd) <= tol * abs(fd) + 1e-5, (k, g["theta"][k], fd)
    r.close()


def test_checkpoint_interval_does_not_change_gradients():
    K = 6
    r, pp, pv, theta = _rbc_rollout(L=(12, 12, 12), seed=41)
    r.set_params(theta)
    out = []
    for kck in (1, 4, 6):
        r.forward(K, kck)
        out.append(r.backward())
    for o in out[1:]:
        np.testing.assert_allclose(o["theta"], out[0]["theta"], rtol=1e-4, atol=1e-9)
        np.testing.assert_allclose(o["gxv"], out[0]["gxv"], rtol=1e-3, atol=1e-7 * np.abs(out[0]["gxv"]).max())
    r.close()


def test_autograd_wrapper_matches_direct_backward():
    from ctc_b200.adjoint import RolloutLoss
    r, pp, pv, theta = _rbc_rollout(L=(12, 12, 12), seed=51)
    th = torch.tensor(theta, dtype=torch.float64, requires_grad=True)
    xs = torch.tensor(pp[:, :3], requires_grad=True)
    xv = torch.tensor(pv[:, :3], requires_grad=True)
    loss = RolloutLoss.apply(r, th, xs, xv, 4, 2)
    loss.backward()
    r.set_params(theta)
    r.set_positions(pp[:, :3], pv[:, :3])
    l2 = r.forward(4, 2)
    g = r.backward()
    assert abs(float(loss.detach()) - l2) <= 1e-6 * max(1.0, abs(l2))
    np.testing.assert_allclose(th.grad.numpy(), g["theta"], rtol=1e-4, atol=1e-10)
    np.testing.assert_allclose(xv.grad.numpy(), g["gxv"], rtol=1e-3, atol=1e-6 * np.abs(g["gxv"]).max())
    assert xs.grad.shape == xs.shape
    r.close()


def _fp64_reference_check(L, ncell, K, kck, seed, spow, params=(0, 1, 2, 3), nvert=3, nsolv=2, hs=(1e-6,),
                          label=""):
    """The adjoint's gradient of the configuration's loss (mean x-velocity of
    the vertices after K steps) against central differences of the FP64 host
    rollout (tests/fp64_rollout.full_rollout: the same dynamics in double,
    stable keys) with steps hs -- for the parameters listed and the initial
    positions of the nvert vertices and nsolv solvent particles with the
    largest gradients.  Returns {component: (adjoint, [differences per h])}."""
    from ctc_b200.adjoint import Rollout
    from tests import fp64_rollout as R
    pp = systems.solvent(L, seed=seed)
    pv, tri, par = systems.rbc_system(L, ncell, seed=seed + 1)
    dpd = list(systems.dpd_params())
    dpd[3] = spow
    fsi = (0.0, 8.0, dpd[2], dpd[3])
    r = Rollout(L, pp, dpd, systems.KBT, systems.DT, pv=pv, tri=tri, rbc=par, fsi=fsi, mmass=systems.RBC_MASS)
    theta = np.array([systems.A_DPD, systems.GAMMA, par["ks"], par["kb"]])
    r.set_params(theta)
    r.forward(K, kck)
    g = r.backward()
    r.close()
    seeds = R.full_seeds(K)
    f32 = lambda x: float(np.float32(x))
    kw = dict(spow=f32(spow), kBT=f32(systems.KBT), dt=f32(systems.DT), mmass=f32(systems.RBC_MASS))

    def loss(th, pp_=pp, pv_=pv):
        _, xv = R.full_rollout(L, pp_, pv_, tri, 642, th, par, fsi, K, seeds, **kw)
        return float(xv[:, 3].mean())

    out = {}
    for k in params:
        fds = []
        for hr in hs:
            h = hr * max(1.0, abs(theta[k]))
            if k >= 2:
                # ks and kb reach the membrane forces as floats (RbcParams):
                # a step of whole float ulps, so that theta +- h is exact
                u = float(np.spacing(np.float32(theta[k])))
                h = u * max(1.0, np.round(h / u))
            tp, tm = theta.copy(), theta.copy()
            tp[k] += h
            tm[k] -= h
            fds.append((loss(tp) - loss(tm)) / (2 * h))
        out[("a", "gamma", "ks", "kb")[k]] = (float(g["theta"][k]), fds)
    for which, arr, gk, cnt in (("vertex", pv, g["gxv"], nvert), ("solvent", pp, g["gx"], nsolv)):
        for f in np.argsort(np.abs(gk).ravel())[::-1][:cnt]:
            i, c = divmod(int(f), 3)
            fds = []
            for h in hs:
                ap, am = arr.astype(np.float64), arr.astype(np.float64)
                ap[i, c] += h
                am[i, c] -= h
                if which == "vertex":
                    fds.append((loss(theta, pp, ap) - loss(theta, pp, am)) / (2 * h))
                else:
                    fds.append((loss(theta, ap, pv) - loss(theta, am, pv)) / (2 * h))
            out["%s %d.%d" % (which, i, c)] = (float(gk[i, c]), fds)
    print(label, {k: "adj %.7e fd %s rel %.2e" % (a, ["%.7e" % x for x in f], abs(a - f[0]) / abs(f[0]))
                  for k, (a, f) in out.items()})
    return out


def test_adjoint_vs_fp64_reference_smooth_weight():
    """Solvent + one red blood cell in a 12^3 box, K = 4, checkpoints every
    2, the pair weight (1 - r)^1: every parameter and the largest position
    gradients within 1e-4 of the FP64 reference (measured: 1e-6 .. 7e-5)."""
    out = _fp64_reference_check((12, 12, 12), 1, 4, 2, seed=61, spow=1.0, label="spow 1")
    for k, (a, f) in out.items():
        assert abs(a - f[0]) <= 1e-4 * abs(f[0]), (k, a, f)


def test_adjoint_vs_fp64_reference_configuration_weight():
    """The same system with the configurations' weight (1 - r)^0.25.  The
    force then has an unbounded slope at the cutoff, and a gradient
    component that a pair close to the cutoff carries is not resolved by
    finite differences of any step: the FP64 differences at steps 1e-6 and
    1e-7 still differ by up to a few percent (the position components with
    the largest gradients are exactly those).  Measured bound: every
    component lies within twice the spread of the two differences plus 2e-4
    of the value; the parameters, whose differences do converge, within 2e-3
    (measured: a 1.1e-3, gamma 7e-4, ks and kb 1.2e-4 -- the FP32 positions
    of pairs within ~1e-6 of the cutoff, where the slope (1 - r)^-0.75 is
    steep, differ from the FP64 ones by rounding, and so do their
    contributions; with the smooth weight above the same code agrees to
    7e-5)."""
    out = _fp64_reference_check((12, 12, 12), 1, 4, 2, seed=61, spow=0.25, hs=(1e-6, 1e-7), label="spow 0.25")
    for k, (a, (f1, f2)) in out.items():
        if k in ("a", "gamma", "ks", "kb"):
            assert abs(a - f2) <= 2e-3 * abs(f2), (k, a, f1, f2)
        else:
            assert abs(a - f2) <= 2 * abs(f1 - f2) + 2e-4 * abs(f2), (k, a, f1, f2)


def test_c4_configuration_gradients_vs_fp64_reference():
    """The C4 configuration itself -- 32^3 at density 10 with 20 cells, K =
    20, checkpoints every 5 -- with the smooth pair weight (1 - r)^1 (the
    kernels take the exponent as a parameter, the code is the same): the four
    parameters and the largest vertex and solvent position gradients within
    1e-4 of the FP64 reference (each FP64 rollout of this size takes seconds
    on the host).  Measured: the parameters 1e-5 .. 6e-5, the positions 4e-6."""
    out = _fp64_reference_check((32, 32, 32), 20, 20, 5, seed=71, spow=1.0, nvert=1, nsolv=1, label="C4")
    for k, (a, f) in out.items():
        assert abs(a - f[0]) <= 1e-4 * abs(f[0]), (k, a, f)
