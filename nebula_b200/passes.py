"""Single reference dispatches on device buffers (the per-pass C ABI).

``PassRunner`` mirrors the reference's per-pass test harness
(tests/helpers/MPMHarness.{h,cpp}: uploadParticles / uploadGrid /
runZeroGrid+runP2G / runGridUpdate / runG2P / runFullStep) over
``nebula_mpm_bin`` / ``_p2g`` / ``_grid_update`` / ``_g2p``.  Device memory is
torch CUDA tensors (plumbing only); every pass is a CUDA kernel in the library.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _capi
from ._capi import call
from .scenes import FIELDS, StepParams


def make_pass(sp: StepParams, n: int) -> _capi.Pass:
    p = _capi.Pass()
    p.dt = sp.dt
    p.cellSize = sp.cell_size
    p.gridRes[:] = list(sp.grid_res)
    p.hashCells = sp.hash_cells
    p.worldMin[:] = list(sp.world_min)
    p.worldMax[:] = list(sp.world_max)
    p.flip_ratio = sp.flip_ratio
    p.particleCount = n
    p.materialCount = len(sp.materials)
    p.colliderCount = len(sp.colliders)
    p.forceCount = len(sp.forces)
    p.mu_lame, p.lambda_lame, p.rho0 = sp.mu_lame, sp.lambda_lame, sp.rho0
    p.M_friction, p.q_cohesion, p.q_max = sp.M_friction, sp.q_cohesion, sp.q_max
    p.plasticModel = sp.plastic_model
    return p


def _vp(t: torch.Tensor | None):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _bytes_tensor(a: np.ndarray, device) -> torch.Tensor:
    b = np.ascontiguousarray(a).view(np.uint8).reshape(-1)
    return torch.from_numpy(b.copy()).to(device)


class PassRunner:
    def __init__(self, sp: StepParams, n: int, device="cuda"):
        self.sp = sp
        self.n = n
        self.dev = torch.device(device)
        nc = sp.hash_cells
        self.nc = nc
        self.state = [torch.zeros((max(n, 1), 4), dtype=torch.float32, device=self.dev) for _ in FIELDS]
        self.grid_mom = torch.zeros((2 * nc, 4), dtype=torch.float32, device=self.dev)
        self.grid_mass = torch.zeros(nc, dtype=torch.float32, device=self.dev)
        self.cell_count = torch.zeros(nc, dtype=torch.int32, device=self.dev)
        self.cell_offset = torch.zeros(nc, dtype=torch.int32, device=self.dev)
        self.sorted = torch.zeros(max(n, 1), dtype=torch.int32, device=self.dev)
        ws = _capi.lib().nebula_mpm_bin_workspace_size(nc, n)
        self.ws = torch.zeros(int(ws), dtype=torch.uint8, device=self.dev)
        self.materials = _bytes_tensor(sp.materials_array(), self.dev)
        self.colliders = _bytes_tensor(sp.colliders_array(), self.dev)
        self.forces = _bytes_tensor(sp.forces_array(), self.dev)
        self.sdf = None

    def _stream(self):
        return C.c_void_p(torch.cuda.current_stream(self.dev).cuda_stream)

    def _parts(self) -> _capi.Particles:
        p = _capi.Particles()
        for k in range(8):
            p.f[k] = self.state[k].data_ptr()
        return p

    def set_params(self, sp: StepParams):
        self.sp = sp
        self.materials = _bytes_tensor(sp.materials_array(), self.dev)
        self.colliders = _bytes_tensor(sp.colliders_array(), self.dev)
        self.forces = _bytes_tensor(sp.forces_array(), self.dev)

    def set_sdf(self, sdf):
        self.sdf = None if sdf is None else torch.from_numpy(np.ascontiguousarray(sdf, np.float32)).to(self.dev)

    def upload_particles(self, st: dict):
        for k, f in enumerate(FIELDS):
            a = torch.from_numpy(np.ascontiguousarray(st[f], np.float32).reshape(-1, 4))
            self.state[k][: a.shape[0]].copy_(a)

    def upload_grid(self, mom, mass):
        m = torch.from_numpy(np.ascontiguousarray(mom, np.float32).reshape(-1, 4))
        self.grid_mom.zero_()
        self.grid_mom[: m.shape[0]].copy_(m)
        self.grid_mass.copy_(torch.from_numpy(np.ascontiguousarray(mass, np.float32)))

    def upload_bins(self, cnt, off, srt):
        self.cell_count.copy_(torch.from_numpy(np.asarray(cnt, np.uint32).view(np.int32)))
        self.cell_offset.copy_(torch.from_numpy(np.asarray(off, np.uint32).view(np.int32)))
        self.sorted[: len(srt)].copy_(torch.from_numpy(np.asarray(srt, np.uint32).view(np.int32)))

    # ------------------------------------------------------------ passes
    def bin(self):
        p = make_pass(self.sp, self.n)
        call("nebula_mpm_bin", C.byref(p), _vp(self.state[0]), _vp(self.cell_count), _vp(self.cell_offset), _vp(self.sorted),
             _vp(self.ws), self.ws.numel(), self._stream())

    def bin_status(self) -> tuple[int, int]:
        """(status code, error bits) of the last bin() on this workspace
        (nebula_mpm_bin_status; synchronizes the stream)."""
        bits = C.c_uint32(0)
        rc = _capi.lib().nebula_mpm_bin_status(_vp(self.ws), self.ws.numel(), self.nc, self.n, C.byref(bits), self._stream())
        return int(rc), int(bits.value)

    def probe_bin_wait_expiry(self):
        """Make the binning scan's bounded look-back expire on this workspace
        (nebula_mpm_bin_probe_wait_expiry); bin_status() then reports bit 1."""
        p = make_pass(self.sp, self.n)
        call("nebula_mpm_bin_probe_wait_expiry", C.byref(p), _vp(self.cell_count), _vp(self.ws), self.ws.numel(), self._stream())

    def p2g(self):
        p = make_pass(self.sp, self.n)
        parts = self._parts()
        call("nebula_mpm_p2g", C.byref(p), C.byref(parts), _vp(self.cell_count), _vp(self.cell_offset), _vp(self.sorted),
             _vp(self.materials), _vp(self.grid_mom), _vp(self.grid_mass), self._stream())

    def grid_update(self):
        p = make_pass(self.sp, self.n)
        call("nebula_mpm_grid_update", C.byref(p), _vp(self.grid_mom), _vp(self.grid_mass), _vp(self.colliders), _vp(self.forces),
             _vp(self.sdf), self._stream())

    def g2p(self):
        p = make_pass(self.sp, self.n)
        parts = self._parts()
        call("nebula_mpm_g2p", C.byref(p), C.byref(parts), _vp(self.grid_mom), _vp(self.grid_mass), _vp(self.materials), _vp(self.sdf),
             self._stream())

    def full_step(self):
        """zero grid, bin, P2G, grid update (+SDF), G2P: one substep."""
        self.bin()
        self.p2g()
        self.grid_update()
        self.g2p()

    # ------------------------------------------------------------ readback
    def read_state(self) -> dict:
        torch.cuda.synchronize(self.dev)
        return {f: self.state[k][: self.n].cpu().numpy().copy() for k, f in enumerate(FIELDS)}

    def read_grid(self):
        torch.cuda.synchronize(self.dev)
        return self.grid_mom.cpu().numpy().copy(), self.grid_mass.cpu().numpy().copy()

    def read_bins(self):
        torch.cuda.synchronize(self.dev)
        return (self.cell_count.cpu().numpy().view(np.uint32).copy(), self.cell_offset.cpu().numpy().view(np.uint32).copy(),
                self.sorted[: self.n].cpu().numpy().view(np.uint32).copy())
