"""Differentiable MPM rollout (``nebula_mpm_adjoint_*``) and a thin
``torch.autograd.Function`` binding over it.

The rollout advances an APIC, ELASTIC (Hencky) body with per-particle Young's
modulus for a fixed number of substeps and returns the loss
|COM(x_T) - target|^2.  Its backward pass is the library's hand-written
adjoint (G2P, grid update, P2G reversed, checkpoints every k substeps); torch
only carries the device buffers.

    roll = Rollout.for_scene(scenes.diff_block())
    v0 = torch.tensor(..., device="cuda", requires_grad=True)
    E = torch.tensor(..., device="cuda", requires_grad=True)
    loss = rollout_loss(roll, x0, v0, E, target)
    loss.backward()          # v0.grad, E.grad from the CUDA adjoint
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _capi
from ._capi import call


def _dptr(t: torch.Tensor | None):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


class Rollout:
    """One differentiable rollout configuration (owns its device buffers)."""

    def __init__(self, domain_size, cell_size, particles, substeps, dt, checkpoint_every=20, gravity=(0.0, -9.8, 0.0), nu=0.3,
                 rho0=1000.0):
        cfg = _capi.AdjointConfig()
        cfg.domainSize[:] = [float(v) for v in domain_size]
        cfg.cellSize = float(cell_size)
        cfg.particles = int(particles)
        cfg.substeps = int(substeps)
        cfg.checkpointEvery = int(checkpoint_every)
        cfg.dt = float(dt)
        cfg.gravity[:] = [float(v) for v in gravity]
        cfg.nu = float(nu)
        cfg.rho0 = float(rho0)
        self.cfg = cfg
        self.n = int(particles)
        h = C.c_void_p()
        call("nebula_mpm_adjoint_create", C.byref(cfg), C.byref(h))
        self._h = h

    @classmethod
    def for_scene(cls, scene, checkpoint_every=None) -> "Rollout":
        sp = scene.params
        ex = scene.extra
        g = np.zeros(3)
        for f in sp.forces:
            g += np.asarray(f["data"][:3], np.float64) * float(f["data"][3])
        return cls(sp.domain_size, sp.cell_size, scene.n, scene.substeps, sp.dt, checkpoint_every or ex.get("checkpoint_every", 20),
                   tuple(g), ex.get("nu", 0.3), ex.get("rho0", sp.rho0))

    def cleanup(self):
        if getattr(self, "_h", None) and self._h.value:
            call("nebula_mpm_adjoint_destroy", self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.cleanup()
        except Exception:
            pass

    # ------------------------------------------------------------ raw calls (device tensors)
    def forward(self, x0: torch.Tensor, v0: torch.Tensor, E: torch.Tensor, target) -> torch.Tensor:
        """x0, v0: (n, 4) float32 CUDA tensors (x, Vp) / (v, -); E: (n,) float32."""
        for t, shape in ((x0, (self.n, 4)), (v0, (self.n, 4)), (E, (self.n,))):
            if not (t.is_cuda and t.dtype == torch.float32 and t.is_contiguous() and tuple(t.shape) == shape):
                raise ValueError("expected a contiguous float32 CUDA tensor of shape %s" % (shape,))
        loss = torch.empty(1, dtype=torch.float32, device=x0.device)
        tgt = (C.c_float * 3)(*[float(v) for v in target])
        call("nebula_mpm_adjoint_forward", self._h, _dptr(x0), _dptr(v0), _dptr(E), tgt, _dptr(loss), _stream())
        return loss[0]

    def backward(self, loss_grad: float = 1.0, want_x0: bool = False):
        dev = torch.device("cuda", torch.cuda.current_device())
        gv = torch.empty((self.n, 4), dtype=torch.float32, device=dev)
        gE = torch.empty(self.n, dtype=torch.float32, device=dev)
        gx = torch.empty((self.n, 4), dtype=torch.float32, device=dev) if want_x0 else None
        call("nebula_mpm_adjoint_backward", self._h, C.c_float(loss_grad), _dptr(gv), _dptr(gE), _dptr(gx), _stream())
        return gv, gE, gx

    def final_state(self, field: str = "P") -> np.ndarray:
        from .engine import FIELD_INDEX
        out = np.empty((self.n, 4), np.float32)
        call("nebula_mpm_adjoint_download", self._h, FIELD_INDEX[field], out.ctypes.data_as(C.c_void_p), out.size)
        return out

    def events(self) -> int:
        e = C.c_uint32()
        call("nebula_mpm_adjoint_events", self._h, C.byref(e))
        return e.value

    def set_graphs(self, enable: bool):
        call("nebula_mpm_adjoint_set_graphs", self._h, int(bool(enable)))

    def launches(self) -> int:
        k = C.c_uint64()
        call("nebula_mpm_adjoint_launches", self._h, C.byref(k))
        return k.value


class RolloutLoss(torch.autograd.Function):
    """loss = |COM(x_T) - target|^2; gradients for v0 (and x0) and E come from
    the CUDA adjoint of the rollout."""

    @staticmethod
    def forward(ctx, x0, v0, E, roll: Rollout, target):
        loss = roll.forward(x0.detach().contiguous(), v0.detach().contiguous(), E.detach().contiguous(), target)
        ctx.roll = roll
        ctx.want_x0 = x0.requires_grad
        return loss

    @staticmethod
    def backward(ctx, g):
        gv, gE, gx = ctx.roll.backward(float(g), want_x0=ctx.want_x0)
        return gx, gv, gE, None, None


def rollout_loss(roll: Rollout, x0: torch.Tensor, v0: torch.Tensor, E: torch.Tensor, target) -> torch.Tensor:
    return RolloutLoss.apply(x0, v0, E, roll, target)
