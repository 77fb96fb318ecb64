"""Block- and tile-size autotuner for the per-substep kernels.

The fused G2P/P2G kernel and the grid update take their launch shape from a
``nebula_mpm_launch_config``: the fused kernel's CTA size (192 or 256 threads),
how many persistent CTAs each of the two kernels keeps per SM, the grid
kernel's nodes per thread per round (2 or 4), and into how many work items
the fused kernel cuts a particle brick (1-4).  Which shape is
fastest depends on the GPU and on the workload (particles per brick, scene
sizes, FLIP or APIC, the material mix), so ``tune`` times candidate shapes on
the caller's own workload with CUDA events and keeps the fastest, by
coordinate descent in three rounds (the fused kernel's CTA shape, its items
per brick, then the grid update's shape), and stores the result in a JSON
cache keyed by the GPU and a
workload key; a later run on the same GPU and workload reuses the entry
without timing anything.  Every shape computes the same substep (float sums
may associate differently), so tuning changes speed, not results.

    shape, report = tune_engine(engine, scene)          # applied to `engine`
    shape, report = tune_batch(batch, scenes, ids)      # applied to `batch`

The cache file is ``$NEBULA_B200_TUNE_CACHE`` if set, else
``~/.cache/nebula_b200/launch_shapes.json``.
"""
from __future__ import annotations

import ctypes as C
import json
import math
import os
import time
from dataclasses import asdict, dataclass, replace
from pathlib import Path
from typing import Callable, Iterable

from . import _capi

CACHE_ENV = "NEBULA_B200_TUNE_CACHE"
CACHE_VERSION = 3  # 2: shapes carry fused_split; 3: 192-thread CTAs, contiguous brick parts


@dataclass(frozen=True)
class LaunchShape:
    fused_threads: int = 0  # 0 = by scene size
    fused_ctas_per_sm: int = 0  # 0 = as many as fit
    grid_ctas_per_sm: int = 0
    grid_batch: int = 4
    fused_split: int = 0  # fused-kernel items per particle brick (0 = by scene size)

    def to_c(self) -> _capi.LaunchConfig:
        return _capi.LaunchConfig(int(self.fused_threads), int(self.fused_ctas_per_sm), int(self.grid_ctas_per_sm), int(self.grid_batch),
                                  int(self.fused_split))

    @staticmethod
    def from_c(c) -> "LaunchShape":
        return LaunchShape(c.fused_threads, c.fused_ctas_per_sm, c.grid_ctas_per_sm, c.grid_batch, c.fused_split)

    @staticmethod
    def coerce(x) -> "LaunchShape":
        if isinstance(x, LaunchShape):
            return x
        if isinstance(x, dict):
            return LaunchShape(**{k: int(v) for k, v in x.items()})
        raise TypeError("a LaunchShape or a dict of its fields")


@dataclass(frozen=True)
class Limits:
    """Most CTAs per SM (occupancy) of each variant: fused[threads == 256], grid[batch == 4]."""
    fused: tuple = (4, 3)
    grid: tuple = (8, 8)

    def fused_max(self, threads: int) -> int:
        return int(self.fused[threads == 256])

    def grid_max(self, batch: int) -> int:
        return int(self.grid[batch == 4])


def device_limits(flip: bool, batch: bool) -> Limits:
    f = (C.c_uint32 * 2)()
    g = (C.c_uint32 * 2)()
    _capi.call("nebula_mpm_launch_limits", int(bool(flip)), int(bool(batch)), f, g)
    return Limits(tuple(f), tuple(g))


def _ctas_options(most: int, extra: Iterable[int]) -> list[int]:
    """0 (= `most`) first, then the other counts below `most`, largest first."""
    out = [0]
    for k in sorted(set(int(e) for e in extra if 1 <= int(e) < most), reverse=True):
        out.append(k)
    return out


def fused_candidates(base: LaunchShape, limits: Limits) -> list[LaunchShape]:
    c = [replace(base, fused_threads=0, fused_ctas_per_sm=0)]  # the engine's choice by scene size
    for threads in (256, 192):
        most = limits.fused_max(threads)
        for k in _ctas_options(most, (most - 1, most // 2)):
            c.append(replace(base, fused_threads=threads, fused_ctas_per_sm=k))
    return c


def split_candidates(base: LaunchShape) -> list[LaunchShape]:
    return [replace(base, fused_split=k) for k in (0, 1, 2, 3, 4)]  # 0: the engine's choice by scene size


def grid_candidates(base: LaunchShape, limits: Limits) -> list[LaunchShape]:
    c = []
    for batch in (4, 2):
        most = limits.grid_max(batch)
        for k in _ctas_options(most, (8, 4, 2)):
            c.append(replace(base, grid_batch=batch, grid_ctas_per_sm=k))
    return c


def cache_path(path=None) -> Path:
    if path is not None:
        return Path(path)
    env = os.environ.get(CACHE_ENV)
    if env:
        return Path(env)
    return Path.home() / ".cache" / "nebula_b200" / "launch_shapes.json"


def _load(path: Path) -> dict:
    try:
        d = json.loads(path.read_text())
        if d.get("version") == CACHE_VERSION and isinstance(d.get("entries"), dict):
            return d
    except (OSError, ValueError):
        pass
    return {"version": CACHE_VERSION, "entries": {}}


def _store(path: Path, key: str, entry: dict) -> None:
    d = _load(path)
    d["entries"][key] = entry
    path.parent.mkdir(parents=True, exist_ok=True)
    tmp = path.with_name(path.name + ".tmp%d" % os.getpid())
    tmp.write_text(json.dumps(d, indent=1, sort_keys=True))
    os.replace(tmp, path)


def workload_key(kind: str, particles: int, cube_res: int, flip: bool, models: Iterable[int], scenes: int = 1) -> str:
    """Particles rounded to a power of two: neighbouring sizes share a shape."""
    p2 = int(round(math.log2(max(1, int(particles)))))
    ms = "-".join(str(int(m)) for m in sorted(set(int(m) for m in models)))
    return "%s|n2^%d|cube%d|%s|models%s|scenes%d" % (kind, p2, int(cube_res), "flip" if flip else "pic-apic", ms, int(scenes))


def device_key() -> str:
    import torch
    p = torch.cuda.get_device_properties(torch.cuda.current_device())
    return "%s|sm%d|cc%d.%d" % (p.name, p.multi_processor_count, p.major, p.minor)


def tune(measure: Callable[[LaunchShape], float], key: str, limits: Limits, path=None, force: bool = False, repeats: int = 2,
         base: LaunchShape = LaunchShape()) -> tuple[LaunchShape, dict]:
    """The fastest shape by `measure` (ms per substep of one shape; called
    `repeats` times per candidate, the minimum kept).  A cached entry under
    `key` is returned unless `force`."""
    p = cache_path(path)
    if not force:
        hit = _load(p)["entries"].get(key)
        if hit is not None:
            return LaunchShape.coerce(hit["shape"]), dict(hit, source="cache", cache=str(p))
    tried: list[tuple[LaunchShape, float]] = []
    seen: dict[LaunchShape, float] = {}

    def timed(s: LaunchShape) -> float:
        if s not in seen:
            seen[s] = min(float(measure(s)) for _ in range(max(1, repeats)))
            tried.append((s, seen[s]))
        return seen[s]

    t_base = timed(base)
    best = min(fused_candidates(base, limits), key=timed)
    best = min(split_candidates(best), key=timed)
    best = min(grid_candidates(best, limits), key=timed)
    entry = {"shape": asdict(best), "ms_per_substep": seen[best], "default_ms_per_substep": t_base,
             "tried": [[asdict(s), t] for s, t in tried], "when": time.strftime("%Y-%m-%dT%H:%M:%S")}
    _store(p, key, entry)
    return best, dict(entry, source="measured", cache=str(p))


def _events_ms(run: Callable[[], None], stream) -> float:
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    run()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def tune_engine(eng, scene, substeps: int = 10, path=None, force: bool = False, repeats: int = 2) -> tuple[LaunchShape, dict]:
    """Tune and apply the shape of `eng` on `scene` (its state is uploaded
    before every candidate and again at the end)."""
    import torch
    sp = scene.params
    flip = sp.flip_ratio > 0.01
    models = [m["model"] for m in sp.materials] if sp.materials else [sp.plastic_model]
    key = device_key() + "|" + workload_key("engine", scene.n, _cube(sp.grid_res), flip, models)
    stream = torch.cuda.Stream()

    def measure(s: LaunchShape) -> float:
        eng.set_launch_config(s)
        eng.upload_state(scene.state)
        eng.run_substeps(sp.dt, 2, stream)  # binning + the pending P2G of a fresh state
        eng.sync()
        return _events_ms(lambda: eng.run_substeps(sp.dt, substeps, stream), stream) / substeps

    shape, rep = tune(measure, key, device_limits(flip, False), path, force, repeats)
    eng.set_launch_config(shape)
    if rep["source"] == "measured":
        eng.upload_state(scene.state)
    return shape, dict(rep, key=key)


def tune_batch(batch, scenes, ids, substeps: int = 20, path=None, force: bool = False, repeats: int = 2) -> tuple[LaunchShape, dict]:
    """Tune and apply the shape of `batch` holding `scenes` as `ids` (their
    states are uploaded before every candidate and again at the end)."""
    import torch
    flip = any(sc.params.flip_ratio > 0.01 for sc in scenes)
    models = [m["model"] for sc in scenes for m in (sc.params.materials or [])] or [0]
    n = sum(sc.n for sc in scenes)
    cube = max(_cube(sc.params.grid_res) for sc in scenes)
    key = device_key() + "|" + workload_key("batch", n, cube, flip, models, len(scenes))
    dt = scenes[0].params.dt
    stream = torch.cuda.Stream()

    def restore():
        for sc, s in zip(scenes, ids):
            batch.upload_state(s, sc.state)

    def measure(s: LaunchShape) -> float:
        batch.set_launch_config(s)
        restore()
        batch.step(dt * substeps, substeps, stream)  # pending P2G, graph capture
        batch.sync()
        return _events_ms(lambda: batch.step(dt * substeps, substeps, stream), stream) / substeps

    shape, rep = tune(measure, key, device_limits(flip, True), path, force, repeats)
    batch.set_launch_config(shape)
    if rep["source"] == "measured":
        restore()
    return shape, dict(rep, key=key)


def _cube(res) -> int:
    m = max(max(res), 1)
    c = 1
    while c < m:
        c <<= 1
    return c
