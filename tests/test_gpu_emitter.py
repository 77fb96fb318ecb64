"""Device-side emission (nebula_mpm_add_emitter) on the GPU.

The particles the emission kernel writes equal the CPU restatement's
(oracle/mpm_emit_oracle.cpp, same counter-based draws); the schedule, the
capacity truncation and the centre motion follow MPMEngine::emitFromEmitters
(MPMEngine.cpp:289-352); and particles emitted into a running, brick-permuted
engine evolve exactly as the same particles appended from the host.
"""
import numpy as np
import pytest

import oracle
from nebula_b200 import scenes as S
from nebula_b200.engine import MPMConfig, MPMEngine, engine_for_scene

pytestmark = pytest.mark.gpu

SEED = 12345


def empty_engine(cap=20000, n_side=20):
    cfg = MPMConfig(nx=n_side, ny=n_side, nz=n_side, domainSize=(1.0, 1.0, 1.0), cellSize=1 / 64, maxParticles=cap, E=1e4, nu=0.3,
                    rho0=1000.0)
    e = MPMEngine(cfg)
    e.resetParticles()
    e.flip_ratio = -1.0
    e.addForce(S.gravity())
    e.numSubsteps = 1
    return e


@pytest.mark.parametrize("em", [
    S.aabb_emitter((0.3, 0.5, 0.3), (0.6, 0.7, 0.5), (0.0, -1.0, 0.0), 3000, particle_type=0),
    S.sphere_emitter((0.5, 0.6, 0.5), 0.15, (1.0, 0.0, 0.0), 3000, along_normal=True, randomness=0.1, particle_type=0),
    S.ellipse_emitter((0.5, 0.6, 0.5), 0.2, 0.1, (0.0, 0.5, 0.0), 3000, particle_type=0),
], ids=["aabb", "sphere_normal_random", "ellipse"])
def test_emitted_particles_match_oracle(em):
    e = empty_engine()
    e.addEmitter(em)
    e.numSubsteps = 0  # emission only
    e.step(1e-3)
    got_p, got_v = e.download("P"), e.download("v")
    Vp = (1.0 / 20) ** 3  # MPMConfig::particleVolume
    want_p, want_v = oracle.emit(em, Vp, SEED, 0, 3000)
    assert got_p.shape == (3000, 4)
    assert np.allclose(got_p, want_p, rtol=0, atol=2e-6)
    assert np.allclose(got_v[:, :3], want_v[:, :3], rtol=0, atol=2e-6)
    assert np.array_equal(got_v[:, 3].view(np.uint32), want_v[:, 3].view(np.uint32))
    F0 = e.download("F0")
    assert np.all(F0 == np.array([1, 0, 0, 0], np.float32))


def test_schedule_truncation_and_motion():
    e = empty_engine(cap=2500, n_side=10)
    once = e.addEmitter(S.aabb_emitter((0.3, 0.5, 0.3), (0.4, 0.6, 0.4), (0, 0, 0), 100, step_count=-1))
    thrice = e.addEmitter(S.aabb_emitter((0.6, 0.5, 0.3), (0.7, 0.6, 0.4), (0, 0, 0), 200, step_count=3))
    always = e.addEmitter(S.sphere_emitter((0.5, 0.3, 0.6), 0.05, (0, 0, 0), 500, step_count=0, center_vel=(0.0, 1.0, 0.0)))
    e.numSubsteps = 2
    counts = []
    for _ in range(6):
        e.step(1e-3)
        counts.append(e.liveParticleCount())
    # step 1: 100+200+500, 2: +200+500, 3: +200+500, 4: +500 -> 2500 (capacity), then nothing more
    assert counts == [800, 1500, 2200, 2500, 2500, 2500]
    rec, done = e.getEmitter(always)
    assert done == 6
    # the centre moved after each of the four emissions that added particles (MPMEngine.cpp:348-350)
    assert np.isclose(rec["center"][1], 0.3 + 4 * 1e-3, atol=1e-6)
    assert e.getEmitter(once)[1] == 1 and e.getEmitter(thrice)[1] == 3
    e.resetParticles()
    assert e.liveParticleCount() == 0 and e.getEmitter(once)[1] == 0
    e.step(1e-3)
    assert e.liveParticleCount() == 800


def test_emission_into_running_engine_equals_host_append():
    """Emit into an engine whose particles are already in brick order (after
    30 fused substeps); the same particles appended from the host give the
    same state after 20 more substeps."""
    sc = S.shear_block()
    cap = sc.n + 2000
    em = S.aabb_emitter((0.3, 0.85, 0.3), (0.5, 0.95, 0.5), (0.0, -0.5, 0.0), 2000, particle_type=0,
                        particle_volume=float(np.float32(0.5 / 64) ** 3))
    a = engine_for_scene(sc, capacity=cap)
    b = engine_for_scene(sc, capacity=cap)
    for eng in (a, b):
        eng.run_substeps(sc.params.dt, 30)
    a.addEmitter(em)
    a.run_substeps(sc.params.dt, 20)  # emits once at the first step() call, then 20 substeps
    pos, vel = oracle.emit(em, float(np.float32(0.5 / 64) ** 3), SEED, 0, 2000)
    assert b.appendParticles(pos, vel) == 2000
    b.run_substeps(sc.params.dt, 20)
    pa, pb = a.download("P"), b.download("P")
    assert pa.shape == (cap, 4)
    err = np.linalg.norm(pa[:, :3] - pb[:, :3]) / np.linalg.norm(pb[:, :3])
    assert err < 1e-5, err  # float atomics order the sums differently in the two engines
