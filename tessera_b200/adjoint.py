"""Differentiable MPM rollout: the device forward with checkpoints and its
hand-written adjoint (``tmpm_adjoint_*`` in include/tmpm.h), exposed to
PyTorch as a ``torch.autograd.Function``.

    sim = Rollout(params, particles, substep_dt=1e-4, substeps=256, checkpoint_every=16)
    x_T = rollout(sim, velocity0, young)          # (N, 3) final positions
    loss = ((x_T.mean(0) - target) ** 2).sum()
    loss.backward()                                # velocity0.grad, young.grad

The forward is the reference substep (crates/tessera-mpm/src/world.rs:361-467)
for corotated elastic particles (material.rs:440-455) in a bounded domain.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native
from ._abi import STATUS_MESSAGES, TMPM_OK, ParticleArrays, TmpmParams
from .session import TesseraError


def _check(status: int, handle=None) -> None:
    if status == TMPM_OK:
        return
    L = _native.lib()
    msg = (L.tmpm_adjoint_last_error_message(handle) if handle else L.tmpm_last_error()) or b""
    raise TesseraError(msg.decode() or STATUS_MESSAGES.get(status, f"status {status}"), status)


def _f64(a, shape):
    if a is None:
        return None
    out = np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(shape))
    return out


class Rollout:
    """A fixed-substep rollout of one scene with its adjoint on the device."""

    def __init__(self, params: TmpmParams, particles: ParticleArrays, substep_dt: float, substeps: int,
                 checkpoint_every: int = 16, device: int = 0):
        handle = C.c_void_p()
        self._h = None
        arrays = particles.as_c()
        _check(_native.lib().tmpm_adjoint_create(C.byref(params), C.byref(arrays), float(substep_dt), int(substeps),
                                                  int(checkpoint_every), int(device), C.byref(handle)))
        self._h = handle
        self.count = particles.count
        self.substeps = int(substeps)
        self.generation = 0  # bumps on every forward; a backward belongs to the latest one

    def close(self) -> None:
        if self._h:
            _native.lib().tmpm_adjoint_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown
            pass

    def forward(self, velocity0=None, young=None):
        """Final (positions, velocities), (N, 3) float64."""
        n = self.count
        v0 = _f64(velocity0, (n, 3))
        E = _f64(young, (n,))
        x = np.empty((n, 3))
        v = np.empty((n, 3))
        _check(_native.lib().tmpm_adjoint_forward(self._h, None if v0 is None else v0.ctypes.data,
                                                   None if E is None else E.ctypes.data, x.ctypes.data, v.ctypes.data),
               self._h)
        self.generation += 1
        return x, v

    def backward(self, position_grad, velocity_grad=None):
        """(dL/dv0 (N, 3), dL/dE (N,)) for the last forward."""
        n = self.count
        xg = _f64(position_grad, (n, 3))
        vg = _f64(velocity_grad, (n, 3))
        gv = np.empty((n, 3))
        gE = np.empty(n)
        _check(_native.lib().tmpm_adjoint_backward(self._h, xg.ctypes.data, None if vg is None else vg.ctypes.data,
                                                    gv.ctypes.data, gE.ctypes.data), self._h)
        return gv, gE


def _function():
    import torch

    class MpmRollout(torch.autograd.Function):
        """x_T = rollout(v0, E); gradients from the device adjoint."""

        @staticmethod
        def forward(ctx, velocity0, young, sim):
            x, _ = sim.forward(velocity0.detach().cpu().double().numpy(), young.detach().cpu().double().numpy())
            ctx.sim = sim
            ctx.generation = sim.generation
            return torch.from_numpy(x).to(device=velocity0.device, dtype=velocity0.dtype)

        @staticmethod
        def backward(ctx, grad_x):
            sim = ctx.sim
            if sim.generation != ctx.generation:
                raise RuntimeError("the rollout ran another forward since this one; its checkpoints are gone")
            gv, gE = sim.backward(grad_x.detach().cpu().double().numpy())
            dev, dt = grad_x.device, grad_x.dtype
            return torch.from_numpy(gv).to(device=dev, dtype=dt), torch.from_numpy(gE).to(device=dev, dtype=dt), None

    return MpmRollout


_FN = None


def rollout(sim: Rollout, velocity0, young):
    """Differentiable final positions of `sim` for initial velocities and Young's moduli (torch tensors)."""
    global _FN
    if _FN is None:
        _FN = _function()
    return _FN.apply(velocity0, young, sim)
