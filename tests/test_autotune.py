"""The launch-shape autotuner (nebula_b200/autotune.py) on the CPU: candidate
sets within the occupancy limits, coordinate descent to the fastest shape of a
synthetic cost, the JSON cache (hit, force, other keys kept, damaged file)."""
import json

from nebula_b200 import autotune as A

LIM = A.Limits(fused=(4, 3), grid=(8, 8))


def test_candidates_stay_within_occupancy():
    f = A.fused_candidates(A.LaunchShape(), LIM)
    assert A.LaunchShape() in f
    for s in f:
        assert s.fused_threads in (0, 192, 256)
        assert s.fused_ctas_per_sm == 0 or 1 <= s.fused_ctas_per_sm < LIM.fused_max(s.fused_threads)
    assert {(s.fused_threads, s.fused_ctas_per_sm) for s in f} == {(0, 0), (256, 0), (256, 2), (256, 1), (192, 0), (192, 3), (192, 2)}
    g = A.grid_candidates(A.LaunchShape(fused_threads=192), LIM)
    assert all(s.fused_threads == 192 for s in g)
    assert {(s.grid_batch, s.grid_ctas_per_sm) for s in g} == {(4, 0), (4, 4), (4, 2), (2, 0), (2, 4), (2, 2)}
    sp = A.split_candidates(A.LaunchShape(fused_threads=192, fused_ctas_per_sm=3))
    assert [s.fused_split for s in sp] == [0, 1, 2, 3, 4] and all(s.fused_ctas_per_sm == 3 for s in sp)
    one = A.Limits(fused=(1, 1), grid=(1, 1))
    assert len(A.fused_candidates(A.LaunchShape(), one)) == 3 and len(A.grid_candidates(A.LaunchShape(), one)) == 2


def cost(s):
    """Fastest at 192 threads, 3 CTAs/SM, 3 items per brick, grid batch 2 with 4 CTAs/SM."""
    c = 10.0
    c += 0.0 if s.fused_threads == 192 else 1.0 if s.fused_threads == 256 else 1.5
    c += {0: 0.5, 3: 0.0, 2: 0.3, 1: 2.0}[s.fused_ctas_per_sm]
    c += 0.0 if s.grid_batch == 2 else 0.1
    c += {0: 0.2, 4: 0.0, 2: 0.05, 8: 0.3}[s.grid_ctas_per_sm]
    c += {0: 0.3, 1: 0.4, 2: 0.1, 3: 0.0, 4: 0.05}[s.fused_split]
    return c


def test_descent_finds_the_cheapest_shape_and_caches_it(tmp_path):
    calls = []

    def measure(s):
        calls.append(s)
        return cost(s)

    path = tmp_path / "shapes.json"
    best, rep = A.tune(measure, "gpu|k", LIM, path, repeats=2)
    assert best == A.LaunchShape(192, 3, 4, 2, 3)
    assert rep["source"] == "measured" and rep["ms_per_substep"] == cost(best)
    assert rep["default_ms_per_substep"] == cost(A.LaunchShape())
    assert len(calls) == 2 * len({s for s in calls})  # every distinct shape timed `repeats` times
    d = json.loads(path.read_text())
    assert d["entries"]["gpu|k"]["shape"] == {"fused_threads": 192, "fused_ctas_per_sm": 3, "grid_ctas_per_sm": 4, "grid_batch": 2,
                                              "fused_split": 3}
    calls.clear()
    best2, rep2 = A.tune(measure, "gpu|k", LIM, path)
    assert best2 == best and rep2["source"] == "cache" and not calls
    A.tune(lambda s: 1.0 if s == A.LaunchShape() else 2.0, "gpu|other", LIM, path)
    d = json.loads(path.read_text())
    assert set(d["entries"]) == {"gpu|k", "gpu|other"}
    assert d["entries"]["gpu|other"]["shape"] == {"fused_threads": 0, "fused_ctas_per_sm": 0, "grid_ctas_per_sm": 0, "grid_batch": 4,
                                                  "fused_split": 0}
    best3, rep3 = A.tune(lambda s: 1.0 if s == A.LaunchShape() else 2.0, "gpu|k", LIM, path, force=True)
    assert best3 == A.LaunchShape() and rep3["source"] == "measured"


def test_damaged_cache_is_replaced(tmp_path):
    path = tmp_path / "shapes.json"
    path.write_text("{not json")
    best, rep = A.tune(cost, "k", LIM, path, repeats=1)
    assert rep["source"] == "measured" and json.loads(path.read_text())["entries"]["k"]["shape"]["fused_threads"] == 192


def test_keys_and_shape_conversions(tmp_path, monkeypatch):
    k = A.workload_key("batch", 3_140_220, 128, False, [2, 0, 2], 64)
    assert k == "batch|n2^22|cube128|pic-apic|models0-2|scenes64"
    assert A.workload_key("engine", 1_000_000, 256, True, [2]) == "engine|n2^20|cube256|flip|models2|scenes1"
    s = A.LaunchShape(192, 4, 2, 2, 3)
    assert A.LaunchShape.from_c(s.to_c()) == s
    assert A.LaunchShape.coerce({"fused_threads": 192, "fused_ctas_per_sm": 4, "grid_ctas_per_sm": 2, "grid_batch": 2, "fused_split": 3}) == s
    assert A.LaunchShape.coerce({"fused_threads": 192}).fused_split == 0
    monkeypatch.setenv(A.CACHE_ENV, str(tmp_path / "x.json"))
    assert A.cache_path() == tmp_path / "x.json"
