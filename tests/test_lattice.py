"""The library's seeded lattice placement (nebula_mpm_lattice_points, host
only) reproduces scenes.jittered_lattice bit for bit: same SplitMix64 stream,
same order of points and axes, same double arithmetic."""
import numpy as np

from nebula_b200 import scenes as S
from nebula_b200.engine import lattice_points, lattice_record


def test_elastic_block_geometry_bit_exact():
    sc = S.elastic_block()
    h = 1.0 / 64
    sp = 0.5 * h
    half = sp * 19 / 2.0
    L = lattice_record((20, 20, 20), sp, (0.5 - half, 0.7 - half, 0.5 - half), 0.25 * h, seed=1, stream=0,
                       particle_volume=float(np.float32(sp) ** 3))
    pos, vel = lattice_points(L)
    assert np.array_equal(pos[:, :3], sc.state["P"][:, :3])
    assert np.array_equal(pos[:, 3], sc.state["P"][:, 3])
    assert np.all(vel == 0.0)


def test_irregular_lattice_bit_exact():
    counts, spacing, origin, jitter = (7, 3, 5), 0.013, (0.1, 0.2333, 0.41), 0.003
    want = S.jittered_lattice(12345, 7, counts, spacing, origin, jitter)
    L = lattice_record(counts, spacing, origin, jitter, seed=12345, stream=7, particle_volume=2e-6, vel=(1.0, -2.0, 0.5), material_id=3)
    pos, vel = lattice_points(L)
    assert pos.shape == (105, 4)
    assert np.array_equal(pos[:, :3], want)
    assert np.all(pos[:, 3] == np.float32(2e-6))
    assert np.all(vel[:, :3] == np.array([1.0, -2.0, 0.5], np.float32))
    assert np.all(vel[:, 3].view(np.uint32) == 3)
    # another stream of the same seed moves every point
    other, _ = lattice_points(lattice_record(counts, spacing, origin, jitter, seed=12345, stream=8))
    assert np.all(np.any(other[:, :3] != pos[:, :3], axis=1))
