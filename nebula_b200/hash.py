"""The PBF fluid engine's spatial hash on the shared counting sort.

FluidEngine::step rebuilds a Morton-ordered spatial hash of the predicted
positions every substep (zero_cells, hash_count, hash_scan_local/global,
hash_add_base, hash_sort; FluidEngine.cpp:445-474) and the pbf_* shaders walk
the 27 neighbour cells of it (pbf_density.comp:44-60).  ``SpatialHash`` owns
the hash buffers and the scan workspace and rebuilds them with one call of
``nebula_hash_bin``, the kernels that bin the MPM particles.

Layout of a PBF particle buffer (FluidEngine.cpp:39-64): slots
[0, max_boundary) hold boundary particles (typeFlag 3) followed by unused
slots (typeFlag 6, predP = 0), which the hash leaves out; fluid particles
follow from max_boundary on.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _capi
from . import scenes as S

TYPE_FLAG_BOUNDARY = 3
TYPE_FLAG_UNUSED = 6


class HashGrid(C.Structure):
    _fields_ = [("worldMin", C.c_float * 3), ("cellSize", C.c_float), ("gridRes", C.c_uint32 * 3), ("hashCells", C.c_uint32)]


@dataclass
class FluidGrid:
    """FluidConfig's hash domain (FluidEngine.h:21-35): gridRes = domain::gridRes
    of (domainSize, cellSize), hashCells = cubeRes^3, worldMin = 0."""
    domain_size: tuple = (20.0, 20.0, 20.0)
    cell_size: float = 20.0 / 64.0
    world_min: tuple = (0.0, 0.0, 0.0)

    @property
    def grid_res(self):
        return S.grid_res(self.domain_size, self.cell_size)

    @property
    def hash_cells(self):
        return S.hash_cells(self.grid_res)

    def to_c(self) -> HashGrid:
        g = HashGrid()
        g.worldMin[:] = [float(v) for v in self.world_min]
        g.cellSize = float(np.float32(self.cell_size))
        g.gridRes[:] = list(self.grid_res)
        g.hashCells = self.hash_cells
        return g


class SpatialHash:
    """cellCount, cellOffset (range ends) and sortedIdx of up to `capacity`
    particles, as torch int32 tensors holding the uint32 bits, on `device`."""

    def __init__(self, grid: FluidGrid, capacity: int, device="cuda"):
        import torch

        self.grid = grid
        self.capacity = int(capacity)
        nc = grid.hash_cells
        self.cell_count = torch.zeros(nc, dtype=torch.int32, device=device)
        self.cell_offset = torch.zeros(nc, dtype=torch.int32, device=device)
        self.sorted_idx = torch.zeros(max(1, self.capacity), dtype=torch.int32, device=device)
        ws = _capi.lib().nebula_hash_bin_workspace_size(nc, self.capacity)
        self.workspace = torch.empty(max(16, ws), dtype=torch.uint8, device=device)
        self._c = grid.to_c()

    def build(self, pred_p, type_flag=None, stream=None):
        """Rebuild from pred_p (n, 4) float32 and type_flag (n,) int32/uint32 or
        None, device tensors with n <= capacity; enqueued on `stream` (default:
        torch's current stream)."""
        import torch

        n = int(pred_p.shape[0])
        if n > self.capacity:
            raise ValueError("%d particles exceed the hash capacity %d" % (n, self.capacity))
        if pred_p.dtype != torch.float32 or not pred_p.is_contiguous() or pred_p.dim() != 2 or pred_p.shape[1] != 4:
            raise ValueError("pred_p must be a contiguous (n, 4) float32 tensor")
        tf = None
        if type_flag is not None:
            if type_flag.shape[0] != n or type_flag.element_size() != 4 or not type_flag.is_contiguous():
                raise ValueError("type_flag must be a contiguous (n,) 32-bit tensor")
            tf = C.c_void_p(type_flag.data_ptr())
        s = stream if stream is not None else torch.cuda.current_stream()
        _capi.call("nebula_hash_bin", C.byref(self._c), C.c_void_p(pred_p.data_ptr()), tf, n, C.c_void_p(self.cell_count.data_ptr()),
                   C.c_void_p(self.cell_offset.data_ptr()), C.c_void_p(self.sorted_idx.data_ptr()), C.c_void_p(self.workspace.data_ptr()),
                   self.workspace.numel(), C.c_void_p(s.cuda_stream))
        return self.cell_count, self.cell_offset, self.sorted_idx


def fluid_layout(seed: int = 7, fluid=(192, 3, 192), grid: FluidGrid | None = None, max_boundary: int = 50000, boundary_used: int = 20000):
    """A FluidEngine particle buffer with the default FluidConfig (192 x 3 x 192
    fluid lattice at spacing domainSize.x / fluid_nx, 50,000 boundary slots on
    a 20 m domain with cellSize 20/64): `boundary_used` boundary particles on
    the floor and two walls (typeFlag 3), the rest of the boundary slots unused
    (typeFlag 6, predP = 0), then the jittered fluid block (typeFlag 0).
    Returns (pred_p (n, 4) float32, type_flag (n,) uint32)."""
    g = grid or FluidGrid()
    L = np.asarray(g.domain_size, np.float64)
    d = L[0] / fluid[0]
    nb = min(boundary_used, max_boundary)
    u = S.uniform(seed, 2 * nb, 3).reshape(nb, 2)
    side = np.arange(nb) % 3  # floor, wall x = 0, wall z = 0
    b = np.zeros((nb, 3))
    b[side == 0] = np.stack([u[side == 0, 0] * L[0], np.full((side == 0).sum(), 0.25 * d), u[side == 0, 1] * L[2]], 1)
    b[side == 1] = np.stack([np.full((side == 1).sum(), 0.25 * d), u[side == 1, 0] * L[1], u[side == 1, 1] * L[2]], 1)
    b[side == 2] = np.stack([u[side == 2, 0] * L[0], u[side == 2, 1] * L[1], np.full((side == 2).sum(), 0.25 * d)], 1)
    fl = S.jittered_lattice(seed, 4, fluid, d, (0.5 * d, 0.5 * d, 0.5 * d), 0.2 * d).astype(np.float64)
    n = max_boundary + fl.shape[0]
    pos = np.zeros((n, 4), np.float32)
    pos[:nb, :3] = b
    pos[max_boundary:, :3] = fl
    pos[:, 3] = 1.0
    pos[nb:max_boundary, 3] = 0.0
    flags = np.zeros(n, np.uint32)
    flags[:nb] = TYPE_FLAG_BOUNDARY
    flags[nb:max_boundary] = TYPE_FLAG_UNUSED
    return pos, flags
