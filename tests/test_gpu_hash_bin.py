"""The PBF spatial hash on the GPU (nebula_hash_bin through SpatialHash),
bit-exact against the CPU oracle: counts, range ends, canonical sortedIdx,
and the untouched tail of sortedIdx past the included particles."""
import numpy as np
import pytest
import torch

import oracle
from nebula_b200 import hash as H

pytestmark = pytest.mark.gpu


def run(grid, p, f, capacity=None):
    hs = H.SpatialHash(grid, capacity or max(1, len(p)))
    hs.sorted_idx.fill_(-1)
    pt = torch.from_numpy(np.ascontiguousarray(p, np.float32).reshape(-1, 4)).cuda()
    ft = None if f is None else torch.from_numpy(f.view(np.int32)).cuda()
    cnt, off, srt = hs.build(pt, ft)
    torch.cuda.synchronize()
    n = len(p)
    return (cnt.cpu().numpy().view(np.uint32), off.cpu().numpy().view(np.uint32), srt.cpu().numpy().view(np.uint32)[:n])


def check(grid, p, f):
    got = run(grid, p, f)
    want = oracle.hash_bin(p, f, grid.world_min, grid.cell_size, grid.grid_res, grid.hash_cells)
    for name, a, b in zip(("cellCount", "cellOffset", "sortedIdx"), got, want):
        assert np.array_equal(a, b), name


def test_fluid_engine_default_layout():
    p, f = H.fluid_layout()
    check(H.FluidGrid(), p, f)


def test_offset_non_cubic_grid_with_clamped_and_nan_positions_no_flags():
    rng = np.random.default_rng(11)
    g = H.FluidGrid(domain_size=(3.0, 1.0, 2.0), cell_size=0.05, world_min=(-1.0, 0.5, 2.0))
    p = np.zeros((50000, 4), np.float32)
    p[:, :3] = rng.uniform(-0.2, 1.2, (50000, 3)) * np.array(g.domain_size) + np.array(g.world_min)
    p[17, 1] = np.nan  # fmax(NaN, 0): that axis lands in cell 0 on both sides
    check(g, p, None)


def test_hash_cells_beyond_the_single_group_scan():
    """2,097,152 hash cells (128^3): past the 1,024 group sums that
    hash_scan_global.comp covers."""
    rng = np.random.default_rng(12)
    g = H.FluidGrid(domain_size=(20.0, 20.0, 20.0), cell_size=20.0 / 128.0)
    n = 1 << 20
    p = np.zeros((n, 4), np.float32)
    p[:, :3] = rng.uniform(0.0, 20.0, (n, 3))
    f = np.where(rng.uniform(size=n) < 0.05, H.TYPE_FLAG_UNUSED, H.TYPE_FLAG_BOUNDARY).astype(np.uint32)
    check(g, p, f)


def test_all_excluded_and_empty():
    g = H.FluidGrid(domain_size=(1.0, 1.0, 1.0), cell_size=0.125)
    p = np.random.default_rng(1).uniform(0, 1, (1000, 4)).astype(np.float32)
    check(g, p, np.full(1000, H.TYPE_FLAG_UNUSED, np.uint32))
    cnt, off, _ = run(g, np.zeros((0, 4), np.float32), None, capacity=16)
    assert not cnt.any() and not off.any()


def test_rebuild_replaces_the_previous_hash():
    g = H.FluidGrid()
    p, f = H.fluid_layout()
    hs = H.SpatialHash(g, len(p))
    pt = torch.from_numpy(p).cuda()
    ft = torch.from_numpy(f.view(np.int32)).cuda()
    hs.build(pt, ft)
    q = p.copy()
    q[:, :3] = q[:, :3][::-1]  # other positions, same flags
    hs.build(torch.from_numpy(np.ascontiguousarray(q)).cuda(), ft)
    torch.cuda.synchronize()
    want = oracle.hash_bin(q, f, g.world_min, g.cell_size, g.grid_res, g.hash_cells)
    assert np.array_equal(hs.cell_count.cpu().numpy().view(np.uint32), want[0])
    assert np.array_equal(hs.cell_offset.cpu().numpy().view(np.uint32), want[1])
    m = int(want[0].sum())
    assert np.array_equal(hs.sorted_idx.cpu().numpy().view(np.uint32)[:m], want[2][:m])
