"""Batched scenes on the GPU (nebula_mpm_batch_*).

The batch has no reference counterpart; its oracle is, per scene, the
single-scene engine (itself checked against the CPU oracle elsewhere) and,
for one scene, the CPU oracle stepped substep by substep with the moving
collider re-set each substep (the reference's re-upload semantics).
"""
import dataclasses

import numpy as np
import pytest
import torch

from nebula_b200 import _capi
from nebula_b200 import scenes as S
from nebula_b200.batch import BatchEngine, batch_for_scenes
from nebula_b200.engine import MPMConfig, engine_for_scene

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def Fm(st):
    return np.concatenate([st["F0"][:, :3], st["F1"][:, :3], st["F2"][:, :3]], axis=1)


def small_mix(n=6, nmax=20000, seed=4):
    return S.batch_mix(seed=seed, n_scenes=n, nmin=2000, nmax=nmax)


def plain_run(sc, substeps, start=0):
    eng = engine_for_scene(sc)
    if sc.params.colliders:
        eng.setColliderTrack(S.collider_track(sc, substeps, start))
    eng.run_substeps(sc.params.dt, substeps)
    return eng.state()


def batch_run(scenes, substeps, graphs=True, steps=1):
    b, ids = batch_for_scenes(scenes)
    b.set_graphs(graphs)
    stream = torch.cuda.Stream()
    for k in range(steps):
        for sc, s in zip(scenes, ids):
            b.set_collider_track(s, S.collider_track(sc, substeps, k * substeps))
        b.run_substeps(scenes[0].params.dt, substeps, stream=stream)
    b.sync()
    return b, ids


def test_batch_matches_plain_per_scene():
    scenes = small_mix()
    b, ids = batch_run(scenes, 40)
    for sc, s in zip(scenes, ids):
        got = b.state(s)
        want = plain_run(sc, 40)
        assert rel_l2(got["P"][:, :3], want["P"][:, :3]) < 1e-5, sc.name
        assert rel_l2(Fm(got), Fm(want)) < 1e-4, sc.name
        assert rel_l2(got["v"][:, :3], want["v"][:, :3]) < 1e-3, sc.name
    st = b.stats()
    assert st["graph_launches"] == 1 and st["error_flags"] == 0 and st["scenes"] == len(scenes)


def test_batch_full_mix_64_scenes():
    """All 64 scenes of the mix (about 2.7M particles, 64^3..128^3 grids) for 10
    substeps; every scene equals its single-scene run."""
    scenes = S.batch_mix()
    b, ids = batch_run(scenes, 10)
    worst = 0.0
    for sc, s in zip(scenes, ids):
        got = b.download(s, "P")[:, :3]
        want = plain_run(sc, 10)["P"][:, :3]
        worst = max(worst, rel_l2(got, want))
    assert worst < 1e-5
    info = [b.scene_info(s) for s in ids]
    assert sum(i["particles"] for i in info) == sum(sc.n for sc in scenes)
    assert all(i["first_brick"] == sum(j["bricks"] for j in info[:k]) for k, i in enumerate(info))


def test_batch_matches_oracle_with_moving_collider():
    """One elastic scene against the CPU oracle, the sphere moved every substep."""
    scenes = [sc for sc in small_mix(n=12, nmax=6000) if sc.params.materials[0]["model"] == S.MAT_ELASTIC][:2]
    assert scenes
    n = 30
    b, ids = batch_run(scenes, n)
    from oracle import Oracle
    for sc, s in zip(scenes, ids):
        o = Oracle("ref32")
        track = S.collider_track(sc, n)
        for k in range(n):
            o.set_params(dataclasses.replace(sc.params, colliders=[track[k, 0]]))
            if k == 0:
                o.set_state(sc.state)
            o.run(1)
        want = o.get_state()
        got = b.state(s)
        assert rel_l2(got["P"][:, :3], want["P"][:, :3]) < 1e-5, sc.name
        assert rel_l2(Fm(got), Fm(want)) < 1e-4, sc.name


def test_graph_replay_equals_eager_odd_substeps():
    """Graph capture/replay and eager launches agree over steps of an odd
    substep count (the ping-pong parity changes between replays)."""
    scenes = small_mix(n=4)
    a, ids = batch_run(scenes, 15, graphs=True, steps=3)
    e, _ = batch_run(scenes, 15, graphs=False, steps=3)
    for s in ids:
        x, y = a.state(s), e.state(s)
        assert rel_l2(x["P"][:, :3], y["P"][:, :3]) < 1e-6
        assert rel_l2(Fm(x), Fm(y)) < 1e-5
    assert a.stats()["graph_launches"] == 3 and e.stats()["graph_launches"] == 0


def test_dt_change_and_host_edits_between_steps():
    """A dt change rebuilds the pending P2G; upload_state and set_params between
    steps take effect as in the single-scene engine."""
    scenes = small_mix(n=3)
    dt = scenes[0].params.dt
    b, ids = batch_for_scenes(scenes)
    stream = torch.cuda.Stream()
    plain = [engine_for_scene(sc) for sc in scenes]
    for sc, s, p in zip(scenes, ids, plain):
        b.set_collider_track(s, S.collider_track(sc, 1))
        p.setColliderTrack(S.collider_track(sc, 1))
    b.run_substeps(dt, 8, stream=stream)
    for p in plain:
        p.run_substeps(dt, 8)
    b.run_substeps(0.5 * dt, 6, stream=stream)
    for p in plain:
        p.run_substeps(0.5 * dt, 6)
    # host edit: replace scene 1's state, switch scene 2 to PIC
    st1 = plain[1].state()
    st1["v"][:, 1] += np.float32(0.25)
    b.upload_state(ids[1], st1)
    plain[1].upload_state(st1)
    b.set_params(ids[2], flip_ratio=0.0)
    plain[2].flip_ratio = 0.0
    b.run_substeps(dt, 7, stream=stream)
    for p in plain:
        p.run_substeps(dt, 7)
    b.sync()
    for s, p in zip(ids, plain):
        got, want = b.state(s), p.state()
        assert rel_l2(got["P"][:, :3], want["P"][:, :3]) < 1e-5
        assert rel_l2(Fm(got), Fm(want)) < 1e-4


def test_batch_errors():
    b = BatchEngine(2, 1000)
    cfg = MPMConfig(nx=0, ny=0, nz=0, domainSize=(1, 1, 1), cellSize=1 / 32, maxParticles=0)
    pos = np.zeros((10, 4), np.float32)
    pos[:, :3] = 0.5
    pos[:, 3] = 1e-6
    vel = np.zeros((10, 4), np.float32)
    s = b.add_scene(cfg, pos, vel)
    with pytest.raises(_capi.NebulaError):
        b.add_scene(cfg, np.zeros((2000, 4), np.float32), np.zeros((2000, 4), np.float32))  # over capacity
    with pytest.raises(_capi.NebulaError):
        b.download(5, "P")  # no such scene
    with pytest.raises(_capi.NebulaError):
        b.upload_state(s, {f: np.zeros((3, 4), np.float32) for f in S.FIELDS})  # wrong count
    b.step(1e-4, 2, stream=torch.cuda.Stream())
    with pytest.raises(_capi.NebulaError):
        b.add_scene(cfg, pos, vel)  # layout fixed after the first step
    b.sync()
    assert b.download(s, "P").shape == (10, 4)


def test_batch_ragged_with_empty_and_single_particle_scenes():
    """Scenes of 0, 1 and 2,000+ particles mixed (an empty scene first and
    last): every non-empty scene equals its single-scene run, empty scenes stay
    empty and the layout tables stay consistent."""
    base = small_mix(3)

    def cut(sc, k):
        return dataclasses.replace(sc, state={f: a[:k].copy() for f, a in sc.state.items()}, name="%s_%d" % (sc.name, k))

    scenes = [cut(base[0], 0), cut(base[1], 1), base[2], cut(base[0], 0), cut(base[1], 7)]
    b, ids = batch_run(scenes, 20)
    info = [b.scene_info(s) for s in ids]
    assert [i["particles"] for i in info] == [sc.n for sc in scenes]
    assert all(i["first_brick"] == sum(j["bricks"] for j in info[:k]) for k, i in enumerate(info))
    for sc, s in zip(scenes, ids):
        got = b.state(s)
        if sc.n == 0:
            assert got["P"].shape == (0, 4)
            continue
        want = plain_run(sc, 20)
        assert rel_l2(got["P"][:, :3], want["P"][:, :3]) < 1e-5, sc.name
    assert b.stats()["error_flags"] == 0
    b.cleanup()


def test_batch_with_flip_and_pic_scenes():
    """FLIP (0.95), PIC (0) and APIC scenes in one batch (the batch then runs
    the FLIP instantiation and keeps a pre-force velocity grid): each scene
    equals its single-scene run."""
    scenes = small_mix(3)
    for sc, fr in zip(scenes, (0.95, 0.0, -1.0)):
        sc.params.flip_ratio = fr
    b, ids = batch_run(scenes, 30)
    for sc, s in zip(scenes, ids):
        got = b.state(s)
        want = plain_run(sc, 30)
        assert rel_l2(got["P"][:, :3], want["P"][:, :3]) < 1e-5, sc.params.flip_ratio
        assert rel_l2(got["v"][:, :3], want["v"][:, :3]) < 1e-3, sc.params.flip_ratio
    b.cleanup()


def test_batch_plastic_models_and_sdf_colliders():
    """Drucker-Prager, granular powder, viscoplastic mud and fluid scenes in one
    batch (the float64 return maps inside the batched kernel), two of them with
    a dense terrain SDF of their own grid: each equals its single-scene run."""
    base = small_mix(4, nmax=8000)
    mats = [S.material(S.MAT_DRUCKER_PRAGER, 3.5e5, 0.3, 1600.0, M_friction=0.6), S.preset_powder(), S.preset_mud(), S.preset_water()]
    scenes = []
    for k, (sc, m) in enumerate(zip(base, mats)):
        sc.params.materials = [m]
        sc.params.rho0 = float(m["rho0"])
        if k % 2 == 0:
            res = sc.params.grid_res[0]
            sc.sdf, _ = S.terrain_sdf(k + 11, res, sc.params.cell_size)
        scenes.append(sc)
    b, ids = batch_run(scenes, 25)
    for sc, s in zip(scenes, ids):
        got = b.state(s)
        want = plain_run(sc, 25)
        assert rel_l2(got["P"][:, :3], want["P"][:, :3]) < 1e-5, sc.name
        assert rel_l2(got["v"][:, :3], want["v"][:, :3]) < 1e-3, sc.name
    b.cleanup()
