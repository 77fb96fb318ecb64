"""The engine's own CUDA-graph replays of the substep loop.

A step whose kernel arguments equal those of the previous step of the same
buffer parity is captured once and replayed after that. A replay must launch
exactly what the uncaptured loop would. So every check here runs two engines
on the same inputs, one with graphs on (the default) and one with graphs off,
and compares their states and their launch counts. The host-side changes
between steps must take effect under replays too: parameters, force table,
dt, colliders, appended particles, launch shape and emitters.
"""
import numpy as np
import pytest

from nebula_b200 import scenes as S
from nebula_b200.engine import engine_for_scene

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def pair(sc, substeps, capacity=None):
    a, b = engine_for_scene(sc, capacity), engine_for_scene(sc, capacity)
    b.set_graphs(False)
    for e in (a, b):
        e.numSubsteps = substeps
    return a, b


def xyz(st, *fields):
    return np.concatenate([st[f][:, :3] for f in fields], axis=1)


def stress6(st):
    return np.stack([st[f][:, 3] for f in ("F0", "F1", "F2", "B0", "B1", "B2")], 1)


def same_state(a, b):
    """Float atomics may order the P2G sums differently from run to run, in
    either engine: x, v and F to 1e-5; the affine B (small differences of grid
    velocities) and the Hencky stress (ill-conditioned for near-equal singular
    values) to 1e-4, as in the oracle parity tests."""
    sa, sb = a.state(), b.state()
    for name, tol, fa, fb in [("x", 1e-5, sa["P"][:, :3], sb["P"][:, :3]), ("v", 1e-5, sa["v"][:, :3], sb["v"][:, :3]),
                              ("F", 1e-5, xyz(sa, "F0", "F1", "F2"), xyz(sb, "F0", "F1", "F2")),
                              ("B", 1e-4, xyz(sa, "B0", "B1", "B2"), xyz(sb, "B0", "B1", "B2")),
                              ("stress", 1e-4, stress6(sa), stress6(sb))]:
        e = rel_l2(fa, fb)
        print("%s rel L2 %.2e" % (name, e))
        assert e < tol, (name, e)


@pytest.mark.parametrize("substeps", [4, 5])
@pytest.mark.parametrize("side_stream", [False, True], ids=["null_stream", "side_stream"])
def test_replays_match_uncaptured_steps(substeps, side_stream):
    """Even substep counts replay from the second step on; odd ones alternate
    the buffer parity and replay from the third."""
    import torch

    sc = S.shear_block()
    a, b = pair(sc, substeps)
    s = torch.cuda.Stream() if side_stream else None
    for _ in range(6):
        a.step(sc.params.dt * substeps, s)
        b.step(sc.params.dt * substeps, s)
    a.sync()
    b.sync()
    ta, tb = a.stats(), b.stats()
    assert ta["graph_launches"] == (5 if substeps % 2 == 0 else 4)
    assert tb["graph_launches"] == 0
    assert ta["kernel_launches"] == tb["kernel_launches"]
    assert ta["substeps"] == tb["substeps"] == 6 * substeps
    same_state(a, b)


def test_host_changes_between_replays():
    """Each change lands in the next step, captured or not."""
    sc = S.shear_block()
    dt = sc.params.dt
    a, b = pair(sc, 4, capacity=sc.n + 500)
    moving = S.shear_block()
    moving.params.colliders = [S.sphere_collider((0.5, 0.25, 0.5), 0.1, vel=(0.0, 0.5, 0.0))]

    def both(fn, steps=3, step_dt=dt * 4):
        for e in (a, b):
            fn(e)
        for _ in range(steps):
            for e in (a, b):
                e.step(step_dt)

    both(lambda e: None)                                                    # replays start
    both(lambda e: e.setForces([S.gravity((0.0, -3.0, 1.0))]))               # table contents
    both(lambda e: setattr(e, "flip_ratio", 0.5))                            # substep parameters
    both(lambda e: None, step_dt=dt * 3)                                     # dt
    both(lambda e: e.setColliderSphere(0.15, 0.5, 0.2, 0.5))                 # SDF contents
    both(lambda e: e.setColliders(moving.params.colliders_array()))         # collider table
    rng = np.random.default_rng(7)
    vp = float(np.float32(0.5 / 64) ** 3)
    pos = np.concatenate([rng.uniform(0.4, 0.6, (500, 3)), np.full((500, 1), vp)], 1).astype(np.float32)
    vel = np.zeros((500, 4), np.float32)
    both(lambda e: e.appendParticles(pos, vel))                              # live count
    both(lambda e: e.set_launch_config({"fused_threads": 192}))              # launch shape
    both(lambda e: setattr(e, "numSubsteps", 6), step_dt=dt * 6)             # substep count
    a.sync()
    b.sync()
    assert a.stats()["graph_launches"] > 8
    assert a.stats()["kernel_launches"] == b.stats()["kernel_launches"]
    same_state(a, b)


def test_collider_track_under_replays():
    """A per-substep collider track (one set per substep) re-uploaded before
    every step: same table pointer, new contents."""
    sc = S.shear_block()
    sc.params.colliders = [S.sphere_collider((0.5, 0.15, 0.5), 0.08, vel=(0.0, 2.0, 0.0))]
    dt = sc.params.dt
    a, b = pair(sc, 4)
    for k in range(6):
        track = S.collider_track(sc, 4, start=4 * k)
        for e in (a, b):
            e.setColliderTrack(track)
            e.step(dt * 4)
    a.sync()
    b.sync()
    assert a.stats()["graph_launches"] >= 4
    same_state(a, b)


def test_emitters_and_switching_graphs_off():
    """Steps that emit change the live count (uncaptured); once the emitter is
    done the loop replays. Switching graphs off drops them mid-run."""
    sc = S.shear_block()
    dt = sc.params.dt
    a, b = pair(sc, 4, capacity=sc.n + 3 * 256)
    em = S.aabb_emitter((0.45, 0.6, 0.45), (0.55, 0.7, 0.55), (0.0, -1.0, 0.0), 256, particle_type=0, step_count=3,
                        particle_volume=float(np.float32(0.5 / 64) ** 3))
    for e in (a, b):
        e.addEmitter(em)
    for _ in range(7):
        for e in (a, b):
            e.step(dt * 4)
    assert a.liveParticleCount() == b.liveParticleCount() == sc.n + 3 * 256
    g = a.stats()["graph_launches"]
    assert g >= 2
    a.set_graphs(False)
    for _ in range(3):
        for e in (a, b):
            e.step(dt * 4)
    assert a.stats()["graph_launches"] == g
    a.set_graphs(True)
    for _ in range(3):
        for e in (a, b):
            e.step(dt * 4)
    assert a.stats()["graph_launches"] == g + 2
    a.sync()
    b.sync()
    same_state(a, b)
