"""Differentiable rollouts over the C ABI (ctc_adj_*): K steps of the solvent
+ membrane system with the random force held fixed by its counter (stable,
id-keyed pair noise) and the reverse pass (hand-written vector-Jacobian
products of the pair and membrane forces, recomputation from checkpoints).

``Rollout`` is the thin ctypes harness; ``RolloutLoss`` puts it behind
``torch.autograd.Function`` so that

    loss = RolloutLoss.apply(rollout, theta, x_solvent, x_vertices)
    loss.backward()

gives d loss / d theta (theta = a, gamma, ks, kb) and d loss / d initial
positions, with loss = mean x-velocity of the membrane vertices after K steps.
"""
import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import CtcError, check, lib

THETA = ("a", "gamma", "ks", "kb")


def _vp(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Rollout:
    """One system (box L, solvent pp, optional membranes pv of template tri)
    and its parameters; dpd = (a, g, s, spow) with s recomputed from g."""

    def __init__(self, L, pp, dpd, kBT, dt, mass=1.0, bodyf=(0.0, 0.0, 0.0), pv=None, tri=None, nv=642,
                 rbc=None, fsi=None, mmass=0.5):
        pp = np.ascontiguousarray(pp, np.float32).reshape(-1, 6)
        cfg = _lib.AdjConfig()
        cfg.LX, cfg.LY, cfg.LZ = (int(x) for x in L)
        cfg.dpd = _lib.DpdParams(*dpd)
        cfg.kBT, cfg.mass, cfg.dt = kBT, mass, dt
        cfg.bodyf = (C.c_float * 3)(*bodyf)
        self.n = len(pp)
        nc, self.nvt = 0, 0
        tri_a = pv_a = None
        rbc_p = fsi_p = None
        if pv is not None and len(pv):
            pv_a = np.ascontiguousarray(pv, np.float32).reshape(-1, 6)
            tri_a = np.ascontiguousarray(tri, np.int32).reshape(-1, 3)
            nc, self.nvt = len(pv_a) // nv, len(pv_a)
            rbc_p = C.byref(_lib.RbcParams(**rbc))
            fsi_p = C.byref(_lib.DpdParams(*fsi))
        self.h = C.c_void_p()
        check(lib().ctc_adj_create(C.byref(cfg), self.n, _vp(pp), nc, nv if nc else 0,
                                   len(tri_a) if nc else 0, _vp(tri_a), _vp(pv_a), rbc_p, fsi_p, float(mmass),
                                   C.byref(self.h)))
        self.pp0, self.pv0 = pp, pv_a

    def close(self):
        if getattr(self, "h", None) and self.h.value and _lib._lib is not None:
            lib().ctc_adj_destroy(self.h)
            self.h = None

    __del__ = close

    def set_params(self, theta):
        t = (C.c_double * 4)(*[float(x) for x in theta])
        check(lib().ctc_adj_set_params(self.h, t))

    def set_positions(self, xs=None, xv=None):
        """Replace the initial positions (velocities kept)."""
        pp = pv = None
        if xs is not None:
            pp = self.pp0.copy()
            pp[:, :3] = np.asarray(xs, np.float32).reshape(-1, 3)
        if xv is not None and self.nvt:
            pv = self.pv0.copy()
            pv[:, :3] = np.asarray(xv, np.float32).reshape(-1, 3)
        check(lib().ctc_adj_set_state(self.h, _vp(pp), _vp(pv)))

    def forward(self, K=20, kck=5, stream=None):
        loss = C.c_double(0)
        check(lib().ctc_adj_forward(self.h, int(K), int(kck), C.byref(loss), _stream(stream)))
        return loss.value

    def final_state(self, stream=None):
        pp = np.zeros((self.n, 6), np.float32)
        pv = np.zeros((self.nvt, 6), np.float32)
        check(lib().ctc_adj_get_final(self.h, _vp(pp), _vp(pv) if self.nvt else None, _stream(stream)))
        return pp, pv

    def backward(self, cot=None, stream=None):
        """Gradients after forward(): of the mean vertex x-velocity, or with
        cot = (cx, cv, cxv, cvv) of sum(cx.x + cv.v) over the final state
        (solvent by particle id).  Returns dict theta, gx, gv, gxv, gvv."""
        gt = (C.c_double * 4)()
        gx = np.zeros((self.n, 3), np.float32)
        gv = np.zeros((self.n, 3), np.float32)
        gxv = np.zeros((self.nvt, 3), np.float32)
        gvv = np.zeros((self.nvt, 3), np.float32)
        outs = (_vp(gx), _vp(gv), _vp(gxv) if self.nvt else None, _vp(gvv) if self.nvt else None)
        if cot is None:
            check(lib().ctc_adj_backward(self.h, gt, *outs, _stream(stream)))
        else:
            cs = [None if c is None else np.ascontiguousarray(c, np.float32) for c in cot]
            check(lib().ctc_adj_backward_cot(self.h, *[_vp(c) for c in cs], gt, *outs, _stream(stream)))
        return {"theta": np.array(gt[:]), "gx": gx, "gv": gv, "gxv": gxv, "gvv": gvv}


def _stream(stream=None):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


class RolloutLoss(torch.autograd.Function):
    """loss = mean x-velocity of the vertices after K steps, as a function of
    theta (4, float64) and the initial solvent / vertex positions:
    ``RolloutLoss.apply(rollout, theta, xs, xv, K, kck)``."""

    @staticmethod
    def forward(ctx, rollout, theta, xs, xv, K=20, kck=5):
        rollout.set_params(theta.detach().cpu().numpy())
        rollout.set_positions(xs.detach().cpu().numpy(), xv.detach().cpu().numpy() if xv is not None else None)
        loss = rollout.forward(K, kck)
        ctx.rollout = rollout
        ctx.meta = (theta.dtype, theta.device, xs.dtype, xs.device)
        return torch.tensor(loss, dtype=torch.float64)

    @staticmethod
    def backward(ctx, gloss):
        g = ctx.rollout.backward()
        tdt, tdev, xdt, xdev = ctx.meta
        s = float(gloss)
        gt = torch.tensor(g["theta"] * s, dtype=tdt, device=tdev)
        gx = torch.tensor(g["gx"] * s, dtype=xdt, device=xdev)
        gxv = torch.tensor(g["gxv"] * s, dtype=xdt, device=xdev) if ctx.rollout.nvt else None
        return None, gt, gx, gxv, None, None
