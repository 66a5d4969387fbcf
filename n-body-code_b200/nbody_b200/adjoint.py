"""Reverse-mode gradients of a fixed-dt Hermite-4 run (nbody_adjoint_*), and
a torch.autograd.Function around them.

    x1, v1 = hermite_rollout(x0, v0, m, eps2=..., dt=..., nsteps=..., checkpoint_every=16)
    loss(x1, v1).backward()        # gradients w.r.t. x0, v0, m

x0, v0 are (3, N) float64 CUDA tensors (rows x, y, z), m is (N,).  The
forward keeps the state every `checkpoint_every` steps; the backward
recomputes each segment and runs the engine's adjoint kernels (pair
acc/jerk VJP in FP64, reverse corrector and predictor).
"""
from __future__ import annotations

import ctypes as C

from . import _lib
from ._lib import check
from .engine import PRECISIONS


class AdjointConfig(C.Structure):
    _fields_ = [("n", C.c_int), ("eps2", C.c_double), ("precision", C.c_int), ("device", C.c_int),
                ("dt", C.c_double), ("nsteps", C.c_int), ("checkpoint_every", C.c_int)]


_vp = C.c_void_p
_SIGS = {
    "nbody_adjoint_create": [C.POINTER(_vp), C.POINTER(AdjointConfig)],
    "nbody_adjoint_destroy": [_vp],
    "nbody_adjoint_forward": [_vp] + [_vp] * 13 + [_vp],
    "nbody_adjoint_backward": [_vp] + [_vp] * 13 + [_vp],
    "nbody_adjoint_vjp_acc_jerk": [_vp] + [_vp] * 20 + [_vp],
}


def _f(name):
    return _lib.bind(name, _SIGS[name])


def _p(t):
    assert t.is_cuda and t.dtype.is_floating_point and t.is_contiguous()
    return _vp(t.data_ptr())


def _rows(t):
    return [t[k] for k in range(t.shape[0])]


class Adjoint:
    """Checkpointed forward + reverse sweep for one (n, eps2, dt, nsteps)."""

    def __init__(self, n: int, eps2: float, dt: float, nsteps: int, checkpoint_every: int = 16,
                 precision: str = "fp64", device: int = 0):
        cfg = AdjointConfig(n, eps2, PRECISIONS[precision], device, dt, nsteps, checkpoint_every)
        h = _vp()
        check(_f("nbody_adjoint_create")(C.byref(h), C.byref(cfg)), "nbody_adjoint_create")
        self._h = h
        self.n, self.eps2, self.dt, self.nsteps = n, eps2, dt, nsteps
        self.checkpoint_every, self.precision, self.device = checkpoint_every, precision, device

    def close(self):
        if getattr(self, "_h", None):
            _f("nbody_adjoint_destroy")(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def forward(self, x, v, m, x1, v1, stream: int):
        check(_f("nbody_adjoint_forward")(self._h, *map(_p, _rows(x)), _p(m), *map(_p, _rows(v)),
                                          *map(_p, _rows(x1)), *map(_p, _rows(v1)), _vp(stream)),
              "nbody_adjoint_forward")

    def backward(self, gx1, gv1, gx0, gv0, gm, stream: int):
        check(_f("nbody_adjoint_backward")(self._h, *map(_p, _rows(gx1)), *map(_p, _rows(gv1)),
                                           *map(_p, _rows(gx0)), *map(_p, _rows(gv0)), _p(gm),
                                           _vp(stream)),
              "nbody_adjoint_backward")

    def vjp_acc_jerk(self, x, v, m, abar, jbar, gx, gv, gm, stream: int):
        check(_f("nbody_adjoint_vjp_acc_jerk")(self._h, *map(_p, _rows(x)), _p(m), *map(_p, _rows(v)),
                                               *map(_p, _rows(abar)), *map(_p, _rows(jbar)),
                                               *map(_p, _rows(gx)), *map(_p, _rows(gv)), _p(gm),
                                               _vp(stream)),
              "nbody_adjoint_vjp_acc_jerk")


def _torch_fn():
    import torch

    class HermiteRollout(torch.autograd.Function):
        @staticmethod
        def forward(ctx, x0, v0, m, adj):
            x0, v0, m = x0.contiguous(), v0.contiguous(), m.contiguous()
            x1 = torch.empty_like(x0)
            v1 = torch.empty_like(v0)
            adj.forward(x0, v0, m, x1, v1, torch.cuda.current_stream(x0.device).cuda_stream)
            ctx.adj = adj
            ctx.shape = (x0.shape, m.shape, x0.device)
            return x1, v1

        @staticmethod
        def backward(ctx, gx1, gv1):
            xs, ms, dev = ctx.shape
            gx1 = torch.zeros(xs, dtype=torch.float64, device=dev) if gx1 is None else gx1.contiguous()
            gv1 = torch.zeros(xs, dtype=torch.float64, device=dev) if gv1 is None else gv1.contiguous()
            gx0 = torch.empty(xs, dtype=torch.float64, device=dev)
            gv0 = torch.empty(xs, dtype=torch.float64, device=dev)
            gm = torch.empty(ms, dtype=torch.float64, device=dev)
            ctx.adj.backward(gx1, gv1, gx0, gv0, gm, torch.cuda.current_stream(dev).cuda_stream)
            return gx0, gv0, gm, None

    return HermiteRollout


_FN = None


def hermite_rollout(x0, v0, m, eps2: float, dt: float, nsteps: int, checkpoint_every: int = 16,
                    precision: str = "fp64", adjoint: Adjoint | None = None):
    """Differentiable fixed-dt Hermite-4 run: returns final (x, v), each (3, N).
    Pass `adjoint` to reuse its device buffers across calls (one rollout in
    flight per Adjoint object: a new forward overwrites its checkpoints)."""
    global _FN
    if _FN is None:
        _FN = _torch_fn()
    n = m.shape[0]
    adj = adjoint or Adjoint(n, eps2, dt, nsteps, checkpoint_every, precision, x0.device.index or 0)
    return _FN.apply(x0, v0, m, adj)
