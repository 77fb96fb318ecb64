"""The PBF spatial hash (oracle/hash_bin_oracle.cpp, nebula_b200/hash.py) on the CPU.

The reference's PBF tests are physics tests (tests/test_pbf.cpp TC1-TC3);
nothing pins the hash arrays themselves, so the oracle is pinned here by a
hand-worked case and by an independent numpy restatement, and the layout
is checked against what the pbf_* shaders read: start = cellOffset -
cellCount and the 27-cell walk (pbf_density.comp:44-60)."""
import ctypes as C

import numpy as np
import pytest

import oracle
from nebula_b200 import _capi
from nebula_b200 import hash as H

SENT = 0xFFFFFFFF


def morton(g):
    def ex(v):
        r = np.zeros_like(v, dtype=np.uint32)
        for b in range(10):
            r |= ((v >> b) & 1).astype(np.uint32) << np.uint32(3 * b)
        return r
    return ex(g[:, 0]) | (ex(g[:, 1]) << np.uint32(1)) | (ex(g[:, 2]) << np.uint32(2))


def numpy_hash(p, flags, wm, cs, res, nc):
    loc = (p[:, :3] - np.asarray(wm, np.float32)) / np.float32(cs)
    loc = np.minimum(np.maximum(loc, np.float32(0)), np.asarray(res, np.float32) - np.float32(1))
    key = morton(loc.astype(np.uint32))
    inc = np.ones(len(p), bool) if flags is None else flags != H.TYPE_FLAG_UNUSED
    cnt = np.bincount(key[inc], minlength=nc).astype(np.uint32)
    end = np.cumsum(cnt).astype(np.uint32)
    order = np.nonzero(inc)[0]
    order = order[np.argsort(key[order], kind="stable")].astype(np.uint32)
    srt = np.full(len(p), SENT, np.uint32)
    srt[: len(order)] = order
    return cnt, end, srt


def test_hand_worked_case():
    p = np.array([[0.5, 0.5, 0.5, 1], [1.5, 0.2, 0.1, 1], [0.1, 1.9, 0.0, 1], [1.2, 1.2, 1.2, 1], [0.3, 0.3, 0.3, 0],
                  [-5.0, 9.0, 0.7, 1], [0.9, 0.1, 0.2, 1], [5.0, 5.0, 5.0, 1]], np.float32)
    flags = np.array([0, 0, 3, 0, 6, 0, 3, 0], np.uint32)
    cnt, off, srt = oracle.hash_bin(p, flags, (0, 0, 0), 1.0, (2, 2, 2), 8)
    assert cnt.tolist() == [2, 1, 2, 0, 0, 0, 0, 2]
    assert off.tolist() == [2, 3, 5, 5, 5, 5, 5, 7]  # range ends (hash_sort consumed the starts)
    assert srt.tolist() == [0, 6, 1, 2, 5, 3, 7, SENT]  # the excluded particle leaves the last slot unwritten


def test_oracle_matches_numpy_on_the_fluid_layout():
    p, f = H.fluid_layout()
    g = H.FluidGrid()
    got = oracle.hash_bin(p, f, g.world_min, g.cell_size, g.grid_res, g.hash_cells)
    want = numpy_hash(p, f, g.world_min, g.cell_size, g.grid_res, g.hash_cells)
    for a, b in zip(got, want):
        assert np.array_equal(a, b)
    assert int(got[0].sum()) == len(p) - int((f == H.TYPE_FLAG_UNUSED).sum())


def test_oracle_matches_numpy_on_a_non_cubic_offset_grid_without_flags():
    rng = np.random.default_rng(3)
    g = H.FluidGrid(domain_size=(3.0, 1.0, 2.0), cell_size=0.05, world_min=(-1.0, 0.5, 2.0))
    p = np.zeros((20000, 4), np.float32)
    p[:, :3] = rng.uniform(-0.2, 1.2, (20000, 3)) * np.array(g.domain_size) + np.array(g.world_min)  # some outside: clamped
    got = oracle.hash_bin(p, None, g.world_min, g.cell_size, g.grid_res, g.hash_cells)
    want = numpy_hash(p, None, g.world_min, g.cell_size, g.grid_res, g.hash_cells)
    for a, b in zip(got, want):
        assert np.array_equal(a, b)


def test_27_cell_walk_finds_every_neighbour():
    """What pbf_density reads: for each particle the 27 cells around its own,
    start = cellOffset - cellCount, give exactly the particles within h."""
    rng = np.random.default_rng(5)
    g = H.FluidGrid(domain_size=(1.0, 1.0, 1.0), cell_size=0.1)
    n = 3000
    p = np.zeros((n, 4), np.float32)
    p[:, :3] = rng.uniform(0.0, 1.0, (n, 3))
    f = np.where(rng.uniform(size=n) < 0.1, H.TYPE_FLAG_UNUSED, 0).astype(np.uint32)
    cnt, off, srt = oracle.hash_bin(p, f, g.world_min, g.cell_size, g.grid_res, g.hash_cells)
    h = np.float32(g.cell_size)
    res = np.array(g.grid_res)
    gi = np.minimum(np.maximum((p[:, :3] / h), 0), res - 1).astype(np.int64)
    inc = f != H.TYPE_FLAG_UNUSED
    for i in rng.choice(np.nonzero(inc)[0], 300, replace=False):
        found = set()
        for d in np.stack(np.meshgrid([-1, 0, 1], [-1, 0, 1], [-1, 0, 1], indexing="ij"), -1).reshape(-1, 3):
            c = gi[i] + d
            if np.any(c < 0) or np.any(c >= res):
                continue
            cid = int(morton(c[None].astype(np.uint32))[0])
            for k in range(int(off[cid] - cnt[cid]), int(off[cid])):
                j = int(srt[k])
                if np.sum((p[i, :3] - p[j, :3]) ** 2) < h * h:
                    found.add(j)
        brute = set(np.nonzero(inc & (np.sum((p[:, :3] - p[i, :3]) ** 2, 1) < h * h))[0].tolist())
        assert found == brute


def test_hash_bin_argument_checks_need_no_gpu():
    g = H.FluidGrid(domain_size=(1.0, 1.0, 1.0), cell_size=0.25).to_c()  # 4^3, hashCells 64
    buf = (C.c_uint32 * 64)()
    a = C.c_void_p(C.addressof(buf))
    ws = _capi.lib().nebula_hash_bin_workspace_size(64, 4)
    assert ws > 0
    bad_cells = H.FluidGrid(domain_size=(1.0, 1.0, 1.0), cell_size=0.25).to_c()
    bad_cells.hashCells = 63
    bad_size = H.FluidGrid(domain_size=(1.0, 1.0, 1.0), cell_size=0.25).to_c()
    bad_size.cellSize = 0.0
    cases = [
        (None, a, 4, a, a, a, a, ws),        # null grid
        (C.byref(bad_cells), a, 4, a, a, a, a, ws),
        (C.byref(bad_size), a, 4, a, a, a, a, ws),
        (C.byref(g), None, 4, a, a, a, a, ws),   # null positions with n > 0
        (C.byref(g), a, 4, None, a, a, a, ws),   # null cellCount
        (C.byref(g), a, 4, a, a, a, a, ws - 1),  # workspace too small
    ]
    for grid, pos, n, cnt, off, srt, wsp, wsb in cases:
        with pytest.raises(_capi.NebulaError):
            _capi.call("nebula_hash_bin", grid, pos, None, n, cnt, off, srt, wsp, wsb, None)
