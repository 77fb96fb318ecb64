"""Emission oracle (oracle/mpm_emit_oracle.cpp) on the CPU: the properties the
reference tests for its emitters (tests/test_mpm.cpp:175-226) -- samples
inside the box, inside the sphere with a volume-uniform mean radius, inside
the ellipse at fixed z -- plus the velocity rules of Emitter::sample_velocity
(src/core/Emitter.h:72-80)."""
import numpy as np

import oracle
from nebula_b200 import scenes as S


def test_aabb_samples_inside_box():
    em = S.emitter(S.EMIT_AABB, (1.0, 2.0, 3.0), (2.0, 4.0, 6.0))
    pos, vel = oracle.emit(em, 1e-6, 12345, 0, 500)
    d = np.abs(pos[:, :3] - np.array([1.0, 2.0, 3.0]))
    assert np.all(d <= np.array([1.0, 2.0, 3.0]) + 1e-5)
    assert np.all(pos[:, 3] == np.float32(1e-6)) and np.all(vel[:, :3] == 0)
    # spread over the whole box, not a corner
    assert np.all(pos[:, :3].std(axis=0) > 0.4 * np.array([1.0, 2.0, 3.0]) / np.sqrt(3))


def test_sphere_samples_inside_radius_volume_uniform():
    em = S.sphere_emitter((0.0, 0.0, 0.0), 2.5, (0, 0, 0), 500)
    pos, _ = oracle.emit(em, 1e-6, 12345, 0, 500)
    r = np.linalg.norm(pos[:, :3], axis=1)
    assert np.all(r <= 2.5 + 1e-4)
    assert 0.5 * 2.5 < r.mean() < 0.95 * 2.5


def test_ellipse_samples_inside_and_fixed_z():
    em = S.ellipse_emitter((1.0, -2.0, 5.0), 3.0, 1.5, (0, 0, 0), 500)
    pos, _ = oracle.emit(em, 1e-6, 12345, 0, 500)
    dx, dy = pos[:, 0] - 1.0, pos[:, 1] + 2.0
    assert np.all(dx * dx / 9.0 + dy * dy / 2.25 <= 1.0 + 1e-5)
    assert np.all(pos[:, 2] == np.float32(5.0))


def test_velocity_rules_and_independent_emissions():
    em = S.sphere_emitter((0.5, 0.5, 0.5), 0.1, (0.0, 2.0, 0.0), 300, along_normal=True, particle_type=3)
    pos, vel = oracle.emit(em, 1e-6, 12345, 4, 300)
    speed = np.linalg.norm(vel[:, :3], axis=1)
    assert np.allclose(speed, 2.0, rtol=1e-5)
    radial = (pos[:, :3] - 0.5) / np.linalg.norm(pos[:, :3] - 0.5, axis=1, keepdims=True)
    assert np.allclose(vel[:, :3] / 2.0, radial, atol=1e-4)
    assert np.all(vel[:, 3].view(np.uint32) == 3)
    em2 = S.aabb_emitter((0, 0, 0), (1, 1, 1), (1.0, 0.0, 0.0), 300, randomness=0.25)
    _, v2 = oracle.emit(em2, 1e-6, 12345, 0, 300)
    assert np.all(np.abs(v2[:, :3] - np.array([1.0, 0.0, 0.0])) <= 0.25 + 1e-6)
    a, _ = oracle.emit(em2, 1e-6, 12345, 0, 300)
    b, _ = oracle.emit(em2, 1e-6, 12345, 1, 300)
    assert np.array_equal(a, oracle.emit(em2, 1e-6, 12345, 0, 300)[0]) and not np.array_equal(a, b)
