"""Committed golden vectors (tests/golden/oracle_fixtures.npz, made by
tests/golden/make_golden.py): the oracle must keep reproducing them (CPU) and
the CUDA engine must match them (GPU)."""
from pathlib import Path

import numpy as np
import pytest

from nebula_b200 import scenes as S

GOLD = np.load(Path(__file__).resolve().parent / "golden" / "oracle_fixtures.npz")


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def oracle_run(sc, n, mode):
    import oracle
    o = oracle.Oracle(mode)
    o.set_params(sc.params)
    o.set_sdf(sc.sdf)
    o.set_state(sc.state)
    if n:
        o.run(n)
    return o


def pack(st, every):
    return np.concatenate([st[f][::every] for f in S.FIELDS], axis=1)


# ----------------------------------------------------------------------------- oracle (CPU)
def test_oracle_bins_golden():
    o = oracle_run(S.elastic_block(), 0, "ref32")
    o.bin()
    cnt, off, srt = o.get_bins()
    nz = np.nonzero(cnt)[0]
    assert np.array_equal(nz, GOLD["bins_cells"])
    assert np.array_equal(cnt[nz], GOLD["bins_count"])
    assert np.array_equal(off[nz], GOLD["bins_end"])
    assert np.array_equal(srt, GOLD["bins_sorted"])


@pytest.mark.parametrize("n", [20, 100])
def test_oracle_shear_golden(n):
    st = oracle_run(S.shear_block(), n, "ref32").get_state()
    assert rel_l2(pack(st, 16), GOLD["shear_ref32_%d" % n]) < 1e-6
    sums = np.array([st[f].astype(np.float64).sum(axis=0) for f in S.FIELDS])
    assert rel_l2(sums, GOLD["shear_ref32_%d_sums" % n]) < 1e-6


def test_oracle_multimaterial_golden():
    st = oracle_run(S.multimaterial(), 20, "mixed").get_state()
    assert rel_l2(st["P"][::80, :3], GOLD["multimaterial_mixed_20_x"]) < 1e-6
    assert rel_l2(st["v"][::80, :3], GOLD["multimaterial_mixed_20_v"]) < 1e-5


# ----------------------------------------------------------------------------- CUDA engine (GPU)
@pytest.mark.gpu
def test_engine_bins_golden():
    from nebula_b200.engine import engine_for_scene
    cnt, off, srt = engine_for_scene(S.elastic_block()).export_bins()
    nz = np.nonzero(cnt)[0]
    assert np.array_equal(nz, GOLD["bins_cells"]) and np.array_equal(cnt[nz], GOLD["bins_count"])
    assert np.array_equal(off[nz], GOLD["bins_end"]) and np.array_equal(srt, GOLD["bins_sorted"])


@pytest.mark.gpu
@pytest.mark.parametrize("pipeline", ["fused", "dense"])
def test_engine_shear_golden(pipeline):
    from nebula_b200.engine import engine_for_scene
    sc = S.shear_block()
    eng = engine_for_scene(sc, pipeline=pipeline)
    eng.run_substeps(sc.params.dt, 20)
    st20 = eng.state()
    eng.run_substeps(sc.params.dt, 80)
    st100 = eng.state()
    for n, st in ((20, st20), (100, st100)):
        g = GOLD["shear_ref32_%d" % n]
        x = pack(st, 16)
        # x and F columns of the packed state (P.xyz, F0..F2.xyz)
        cols = [0, 1, 2, 8, 9, 10, 12, 13, 14, 16, 17, 18]
        e = rel_l2(x[:, cols], g[:, cols])
        print("%s shear golden %d substeps: x,F rel L2 %.2e" % (pipeline, n, e))
        assert e < 1e-4


@pytest.mark.gpu
def test_engine_multimaterial_golden():
    from nebula_b200.engine import engine_for_scene
    sc = S.multimaterial()
    eng = engine_for_scene(sc)
    eng.run_substeps(sc.params.dt, 20)
    st = eng.state()
    assert rel_l2(st["P"][::80, :3], GOLD["multimaterial_mixed_20_x"]) < 1e-5
    assert rel_l2(st["v"][::80, :3], GOLD["multimaterial_mixed_20_v"]) < 1e-3
