"""Launch shapes on the GPU: every shape the autotuner may pick computes the
same substep as the default (engine and batch, APIC and FLIP), bad shapes are
rejected, and tune_engine / tune_batch apply and cache their choice."""
import numpy as np
import pytest

from nebula_b200 import _capi
from nebula_b200 import autotune as A
from nebula_b200 import scenes as S
from nebula_b200.batch import batch_for_scenes
from nebula_b200.engine import engine_for_scene

pytestmark = pytest.mark.gpu

SHAPES = [A.LaunchShape(), A.LaunchShape(192, 0, 0, 4), A.LaunchShape(256, 1, 2, 2), A.LaunchShape(192, 3, 4, 2), A.LaunchShape(256, 2, 8, 4),
          A.LaunchShape(256, 0, 0, 4, 4), A.LaunchShape(256, 0, 0, 4, 2), A.LaunchShape(192, 0, 0, 4, 3)]


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("flip", [-1.0, 0.95])
def test_every_shape_computes_the_same_substeps(flip):
    sc = S.shear_block(S.MAT_ELASTIC, flip_ratio=flip)
    ref = None
    for shape in SHAPES:
        e = engine_for_scene(sc)
        e.set_launch_config(shape)
        assert e.launch_config() == shape
        e.run_substeps(sc.params.dt, 30)
        st = e.state()
        e.cleanup()
        if ref is None:
            ref = st
            continue
        assert rel(st["P"][:, :3], ref["P"][:, :3]) < 1e-6, shape
        assert rel(st["v"][:, :3], ref["v"][:, :3]) < 1e-4, shape
        assert rel(st["F0"][:, :3], ref["F0"][:, :3]) < 1e-5, shape


def test_bad_shapes_are_rejected():
    e = engine_for_scene(S.shear_block())
    for bad in (A.LaunchShape(64, 0, 0, 4), A.LaunchShape(128, 0, 0, 4), A.LaunchShape(256, 0, 0, 3), A.LaunchShape(256, 65, 0, 4), A.LaunchShape(256, 0, 0, 4, 5)):
        with pytest.raises(_capi.NebulaError):
            e.set_launch_config(bad)
    assert e.launch_config() == A.LaunchShape()
    lim = A.device_limits(False, False)
    assert lim.fused_max(256) >= 1 and lim.fused_max(192) >= lim.fused_max(256) and lim.grid_max(4) >= 1


def test_batch_shapes_agree_and_tune_batch_caches(tmp_path):
    scenes = S.batch_mix(only={0, 1, 2, 3})
    out = []
    for shape in (A.LaunchShape(), A.LaunchShape(192, 0, 4, 2), A.LaunchShape(256, 0, 0, 4, 3)):
        b, ids = batch_for_scenes(scenes)
        b.set_launch_config(shape)
        assert b.launch_config() == shape
        b.step(scenes[0].params.dt * 20, 20)
        out.append([b.download(s, "P")[:, :3] for s in ids])
        b.cleanup()
    for other in out[1:]:
        for a, c in zip(other, out[0]):
            assert rel(a, c) < 1e-6
    b, ids = batch_for_scenes(scenes)
    path = tmp_path / "shapes.json"
    shape, rep = A.tune_batch(b, scenes, ids, substeps=5, path=path, repeats=1)
    assert rep["source"] == "measured" and b.launch_config() == shape
    assert rep["ms_per_substep"] <= rep["default_ms_per_substep"]
    shape2, rep2 = A.tune_batch(b, scenes, ids, substeps=5, path=path)
    assert rep2["source"] == "cache" and shape2 == shape
    b.cleanup()


def test_tune_engine_applies_restores_and_caches(tmp_path):
    sc = S.shear_block(S.MAT_DRUCKER_PRAGER)
    e = engine_for_scene(sc)
    path = tmp_path / "shapes.json"
    shape, rep = A.tune_engine(e, sc, substeps=5, path=path, repeats=1)
    assert rep["source"] == "measured" and e.launch_config() == shape and len(rep["tried"]) >= 6
    assert np.array_equal(e.download("P"), sc.state["P"])  # state restored after tuning
    shape2, rep2 = A.tune_engine(e, sc, path=path)
    assert rep2["source"] == "cache" and shape2 == shape
