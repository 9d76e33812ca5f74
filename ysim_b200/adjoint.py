"""Differentiable cloth rollouts: the CUDA adjoint wrapped as a
torch.autograd.Function.

    roll = ClothRollout(spec, steps=200, checkpoint_every=20)
    xT = roll(k, L, v0)            # k, L: (S,) float32 CUDA; v0: (V, 3) float32 CUDA
    loss = ((xT - target) ** 2).sum(1).mean()
    loss.backward()                # k.grad, L.grad, v0.grad via ys_adjoint_backward

The forward pass is `steps` fused substeps of the scene (the same kernels as
Simulator::update's substep loop) with checkpoints every `checkpoint_every`
substeps; the backward pass replays each segment and runs the hand-written
reverse kernels (springs, semi-implicit integration, contact projection with
the forward's active set).  Gradients are w.r.t. per-spring stiffness, rest
length (canonical spring order, see generators.grid_spring_params) and the
cloth's initial velocity.

    roll = ClothRollout(spec, steps=200, precision=64)
    xT = roll(k64, L64, v064)      # float64 tensors: binary64 in and out

precision=64 runs the rollout and its reverse pass in binary64 (the FP64
reference rollout's operations; the gradients then agree with FP64 finite
differences), float32 tensors are widened and the results rounded.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib
from .generators import SceneSpec
from .scene import Scene


class _Fn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, k, L, v0, roll):
        xT = roll._forward(k, L, v0)
        ctx.roll = roll
        return xT

    @staticmethod
    def backward(ctx, gx):
        gk, gL, gv = ctx.roll._backward(gx)
        return gk, gL, gv, None


class ClothRollout:
    def __init__(self, spec: SceneSpec, steps: int, checkpoint_every: int = 20, device: int = 0,
                 precision: int = 32, tree_layout=None):
        self.scene = Scene(spec, device=device, tree_layout=tree_layout)
        self.lib = self.scene.lib
        self.device = torch.device("cuda", device)
        self.nV = spec.meshes[0].nV
        h = C.c_void_p()
        _lib.check(self.lib.ys_adjoint_create(C.byref(h), self.scene.h, 0, steps, checkpoint_every),
                   "ys_adjoint_create")
        self.h = h
        self.S = int(self.lib.ys_adjoint_num_springs(self.h))
        self.steps = steps
        self.precision = precision
        self._f64 = False  # the last forward took binary64 tensors
        if precision != 32:
            _lib.check(self.lib.ys_adjoint_set_precision(self.h, precision), "ys_adjoint_set_precision")

    def close(self):
        if getattr(self, "h", None):
            self.lib.ys_adjoint_destroy(self.h)
            self.h = None
        self.scene.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _p(t):
        return C.c_void_p(t.data_ptr())

    def _sync_torch(self):
        torch.cuda.current_stream(self.device).synchronize()

    def _forward(self, k, L, v0):
        self._f64 = self.precision == 64 and k.dtype == torch.float64
        if self._f64:
            k, L, v0 = (t.detach().contiguous().double() for t in (k, L, v0))
            assert k.numel() == self.S and L.numel() == self.S and v0.numel() == 3 * self.nV
            self._sync_torch()
            _lib.check(self.lib.ys_adjoint_set_params_f64(self.h, self._p(k), self._p(L), self._p(v0)),
                       "set_params_f64")
            xT = torch.empty((self.nV, 3), dtype=torch.float64, device=self.device)
            _lib.check(self.lib.ys_adjoint_forward_f64(self.h, self._p(xT)), "ys_adjoint_forward_f64")
            return xT
        k = k.detach().contiguous().float()
        L = L.detach().contiguous().float()
        v0 = v0.detach().contiguous().float()
        assert k.numel() == self.S and L.numel() == self.S and v0.numel() == 3 * self.nV
        self._sync_torch()
        _lib.check(self.lib.ys_adjoint_set_params(self.h, self._p(k), self._p(L), self._p(v0)), "set_params")
        xT = torch.empty((self.nV, 3), dtype=torch.float32, device=self.device)
        _lib.check(self.lib.ys_adjoint_forward(self.h, self._p(xT)), "ys_adjoint_forward")
        self.scene.sync()
        return xT

    def _backward(self, gx):
        if self._f64:
            gx = gx.contiguous().double()
            gk = torch.empty(self.S, dtype=torch.float64, device=self.device)
            gL = torch.empty(self.S, dtype=torch.float64, device=self.device)
            gv = torch.empty((self.nV, 3), dtype=torch.float64, device=self.device)
            self._sync_torch()
            _lib.check(self.lib.ys_adjoint_backward_f64(self.h, self._p(gx), self._p(gk), self._p(gL), self._p(gv)),
                       "ys_adjoint_backward_f64")
            return gk, gL, gv
        gx = gx.contiguous().float()
        gk = torch.empty(self.S, dtype=torch.float32, device=self.device)
        gL = torch.empty(self.S, dtype=torch.float32, device=self.device)
        gv = torch.empty((self.nV, 3), dtype=torch.float32, device=self.device)
        self._sync_torch()
        _lib.check(self.lib.ys_adjoint_backward(self.h, self._p(gx), self._p(gk), self._p(gL), self._p(gv)),
                   "ys_adjoint_backward")
        return gk, gL, gv

    def __call__(self, k, L, v0):
        return _Fn.apply(k, L, v0, self)
