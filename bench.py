#!/usr/bin/env python3
"""Benchmark of the MPMEngine substep on B200 (one JSON line on rank 0).

Workload (default): the 1,000,000-particle Drucker-Prager slope over a 256^3
terrain SDF (seeded synthetic scene; APIC, dt = 2e-5).  One bench "step" is one
MPMEngine::step call of ``--substeps`` substeps.  ``value`` is the whole-job
particle-substeps/s with the state resident in HBM, timed by CUDA events on the
engine's stream (max over ranks); ``e2e`` is the same metric through the C ABI
with the particle state copied host->device before and device->host after every
step.  ``--impl reference`` times the reference's own MPM shaders compiled for
the host cores (``oracle/_ref``; the CPU oracle restating them where that
library is absent) on the same workload.

Multi-GPU: the single scene does not shard; each rank runs a replica
(weak scaling, no collective on the data path).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "particle-substeps/sec/GPU, plain vs batched; adjoint step time; % of HBM peak"
UNIT = "particle-substeps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20, help="timed steps (default 20 x 25 substeps = the workload's 500 substeps)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="nebula", choices=["nebula", "reference"])
    ap.add_argument("--workload", default="slope", choices=["slope", "elastic", "multimaterial"])
    ap.add_argument("--substeps", type=int, default=25,
                    help="substeps per step() call; the timed steps run substeps 1 .. steps * substeps of the workload "
                         "(default 20 x 25 = the 500 substeps of the slope scene)")
    ap.add_argument("--pipeline", default="fused", choices=["fused", "dense"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample-substeps", type=int, default=0, help="oracle substeps timed for cpu_baseline (0 = auto)")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-vs-plain measurement on the 64-scene mix")
    ap.add_argument("--batch-steps", type=int, default=10,
                    help="timed steps of 20 substeps of the batched / plain comparison (10 = the mix's 200 substeps)")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint-vs-forward measurement")
    ap.add_argument("--no-mesh-sdf", action="store_true", help="skip the mesh -> SDF build measurement")
    ap.add_argument("--no-tune", action="store_true", help="default launch shapes instead of the autotuner's")
    ap.add_argument("--mesh-sdf-only", action="store_true", help="only the mesh -> SDF build measurement (one JSON line)")
    return ap.parse_args()


def make_scene(name):
    """The workload from nebula_b200/configs.json: slope = cfg3, elastic = cfg1, multimaterial = cfg2."""
    from nebula_b200 import scenes as S
    return S.load_config({"slope": "cfg3", "elastic": "cfg1", "multimaterial": "cfg2"}[name])


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    """SM clock and throttle-reason sampling during the timed region.

    Polls NVML every 5 ms from a thread on the device the bench runs on
    (matched by UUID); falls back to ``nvidia-smi -lms 200`` when NVML is not
    importable.  Read-only: no clock or power setting is touched."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.thread = None
        self.sm, self.smax, self.reasons = [], [], set()
        self.path = Path("/tmp/nebula_clocks_%d_%d.csv" % (os.getpid(), index))

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        try:
            uuid = str(torch.cuda.get_device_properties(self.index).uuid)
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def start(self):
        try:
            nv, h = self._nvml_handle()
        except Exception:
            nv = None
        if nv is not None:
            bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown, "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                    "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown, "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
            self.stop_flag = threading.Event()
            smax = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)

            def poll():
                while not self.stop_flag.is_set():
                    try:
                        self.sm.append(float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)))
                        self.smax.append(float(smax))
                        r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                        self.reasons.update(k for k, b in bits.items() if r & b)
                    except Exception:
                        pass
                    time.sleep(0.005)

            self.thread = threading.Thread(target=poll, daemon=True)
            self.thread.start()
            return
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self) -> dict:
        if self.thread is not None:
            self.stop_flag.set()
            self.thread.join(timeout=5)
            src = "nvml"
        elif self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            for line in self.path.read_text().splitlines():
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    self.sm.append(float(parts[1]))
                    self.smax.append(float(parts[2]))
                except ValueError:
                    continue
                for nm, val in zip(self.NAMES, parts[5:9]):
                    if val.lower().startswith("active"):
                        self.reasons.add(nm)
            try:
                self.path.unlink()
            except OSError:
                pass
            src = "nvidia-smi"
        else:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no NVML or nvidia-smi"]}
        sm = self.sm
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(self.smax) if self.smax else None,
                "sm_min_mhz": min(sm) if sm else None, "reasons": sorted(self.reasons), "samples": len(sm), "source": src}


# ----------------------------------------------------------------------------- algorithmic bytes
def algorithmic_bytes(phase: str, n: int, active: int, nc: int, flip: bool, sdf: bool) -> float:
    """Minimal DRAM bytes one launch of each phase must move: per particle its
    state read and written once (x, v, F, B: 96 B written, those plus the
    volume and material id: 104 B read) and 8 B of bin key and rank; per active
    node 16 B accumulated by P2G, 16 B read and 16 B written by the grid update
    and 16 B read by G2P; FLIP and the particle SDF check add their reads."""
    a = active
    if phase == "g2p":
        b = n * (80 + 128) + a * 20
        if flip:
            b += 16 * a + 0 * n
        if sdf:
            b += 4 * n
        return float(b)
    if phase == "g2p2g":
        b = 208 * n + 64 * a
        if flip:
            b += 12 * n + 32 * a
        if sdf:
            b += 4 * a + 4 * n
        return float(b)
    if phase == "p2g":
        return float(n * 132 + a * 16)
    if phase == "grid":
        return float(nc * 4 + a * 48 + (4 * a if sdf else 0))
    if phase == "bin":
        return float(52 * n + 12 * nc)
    return 0.0


def canonical_bytes(n, active, flip, sdf):
    """Per-substep canonical algorithmic bytes: 208 N + 64 A (+FLIP, +SDF adders)."""
    b = 208 * n + 64 * active
    if flip:
        b += 12 * n + 32 * active
    if sdf:
        b += 4 * active + 4 * n
    return float(b)


# ----------------------------------------------------------------------------- reference arm
def cpu_reference(sc):
    """The CPU implementation of the reference's substep on this host: its own
    MPM shaders compiled for the CPU (``oracle/_ref``, built by
    ``oracle/build_ref.py``; the independent per-invocation passes spread over
    the host threads; the binning's scan passes give the exclusive prefix they
    intend, so that the trajectory is a correct one at any grid size) when that
    library is present, else the CPU oracle that restates them (identical
    results, ``tests/test_ref_shaders.py``).
    Returns (runner, kind, threads, description)."""
    import oracle
    threads = oracle.num_threads()
    try:
        from oracle import ref as R
        if R.available(prebuilt=True):
            r = R.RefShaders(threads, intended_scan=True)
            r.set_params(sc.params)
            r.set_sdf(sc.sdf)
            r.set_state(sc.state)
            return r, "reference", threads, ("the reference's MPM shaders compiled for the CPU (oracle/_ref), OpenMP, "
                                             "with the binning scan's intended exclusive prefix (the reference's "
                                             "one-workgroup global scan is wrong above 262,144 cells)")
    except OSError:
        pass
    o = oracle.Oracle("ref32")
    o.set_params(sc.params)
    o.set_sdf(sc.sdf)
    o.set_state(sc.state)
    return o, "port", threads, "CPU oracle ref32 mode, OpenMP"


def run_reference(args, rank, world):
    if rank != 0:
        return
    sc = make_scene(args.workload)
    o, kind, cores, what = cpu_reference(sc)
    for _ in range(args.warmup):
        o.substep()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        o.substep()
    dt = time.perf_counter() - t0
    v = sc.n * args.steps / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded)",
        "config": {"workload": sc.name, "particles": sc.n, "grid": list(sc.params.grid_res), "substeps_per_step": 1,
                   "note": "each step is one substep of the workload (a bounded sample); the reference's shaders have no "
                           "graphics API to run through on the box, so they run compiled for the host cores: " + what},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": kind,
                         "sample": "%d substeps of %s after %d warm-up, %s" % (args.steps, sc.name, args.warmup, what)},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- batched vs plain
def measure_batch(steps: int, warmup: int, substeps: int, dist=None, tune: bool = True) -> dict:
    """The 64-scene mix advanced by the batched engine (one set of launches
    per substep, replayed from a CUDA graph) and by single-scene engines
    stepped one after another, on the same stream, with each scene's moving
    sphere re-uploaded as a collider track before every step in both forms.
    With several ranks the scenes are partitioned by particle count
    (nebula_b200.shard); each rank runs its share and the time is the maximum
    over ranks (the total work is fixed: strong scaling)."""
    import torch

    from nebula_b200 import scenes as S
    from nebula_b200 import shard
    from nebula_b200.batch import batch_for_scenes
    from nebula_b200.engine import engine_for_scene

    rank, world, _ = shard.rank_info()
    sizes = S.batch_mix_sizes()
    mine = shard.partition_scenes(sizes, world)[rank]
    scenes = S.batch_mix(only=set(mine))
    n_all = sum(sizes)
    dt = scenes[0].params.dt
    frames = max(warmup, steps)
    tracks = [[S.collider_track(sc, substeps, k * substeps) for k in range(frames)] for sc in scenes]
    stream = torch.cuda.Stream()

    def timed(step_fn, restart):
        # warm-up steps from the initial states, then the initial states again:
        # the timed steps cover substeps 1 .. steps * substeps of the mix
        for k in range(warmup):
            step_fn(k)
        torch.cuda.synchronize()
        restart()
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for k in range(steps):
            step_fn(k)
        e1.record(stream)
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        return shard.max_over_ranks(e0.elapsed_time(e1), dist, "cuda")

    b, ids = batch_for_scenes(scenes)
    tuned = None
    if tune:
        from nebula_b200 import autotune
        _, rep = autotune.tune_batch(b, scenes, ids, substeps=substeps)
        tuned = {"shape": rep["shape"], "source": rep["source"], "ms_per_substep": rep["ms_per_substep"],
                 "default_ms_per_substep": rep["default_ms_per_substep"], "shapes_tried": len(rep["tried"]), "key": rep["key"]}

    def batch_step(k):
        for i, s in enumerate(ids):
            b.set_collider_track(s, tracks[i][k])
        b.step(dt * substeps, substeps, stream)

    def batch_restart():
        for i, s in enumerate(ids):
            b.upload_state(s, scenes[i].state)

    st0 = b.stats()
    ms_b = timed(batch_step, batch_restart)
    b.sync()
    st1 = b.stats()
    launches_b = int(st1["kernel_launches"] - st0["kernel_launches"])
    b.cleanup()

    engines = [engine_for_scene(sc) for sc in scenes]
    for e in engines:
        e.numSubsteps = substeps

    def plain_step(k):
        for i, e in enumerate(engines):
            e.setColliderTrack(tracks[i][k])
            e.step(dt * substeps, stream)

    def plain_restart():
        for i, e in enumerate(engines):
            e.upload_state(scenes[i].state)

    l0 = sum(e.stats()["kernel_launches"] for e in engines)
    ms_p = timed(plain_step, plain_restart)
    for e in engines:
        e.sync()
    launches_p = int(sum(e.stats()["kernel_launches"] for e in engines) - l0)
    for e in engines:
        e.cleanup()
    ps = float(n_all) * substeps * steps
    return {"workload": "batch_mix_64", "scenes": len(sizes), "particles": n_all, "substeps_per_step": substeps, "steps": steps,
            "substep_range": [1, steps * substeps],
            "warmup": warmup, "dt": dt, "value": ps / (ms_b * 1e-3), "ms_per_step": ms_b / steps, "plain_value": ps / (ms_p * 1e-3),
            "plain_ms_per_step": ms_p / steps, "speedup": ms_p / ms_b, "unit": UNIT, "gpu_launches": launches_b,
            "plain_gpu_launches": launches_p, "n_gpus": world, "scaling": "strong" if world > 1 else "single",
            "scenes_on_rank0": len(mine), "autotune": tuned,
            "note": "batched: one grid update + one fused G2P/P2G + scan + permutation per substep over all scenes, graph "
                    "replay; plain: the same kernels per scene, one engine per scene in sequence; ranks take scenes by a "
                    "particle-balanced greedy partition, time = max over ranks"}


# ----------------------------------------------------------------------------- adjoint
def measure_adjoint(steps: int, warmup: int) -> dict:
    """Forward rollout (with checkpoints) and its reverse pass on the
    differentiable 50,000-particle workload, each replayed from a CUDA graph,
    timed with CUDA events on one stream; the single-scene engine's forward on
    the same scene (uniform E) is timed beside it."""
    import torch

    from nebula_b200 import scenes as S
    from nebula_b200.adjoint import Rollout
    from nebula_b200.engine import engine_for_scene

    sc = S.diff_block()
    roll = Rollout.for_scene(sc)
    side = torch.cuda.Stream()
    x0 = torch.from_numpy(sc.state["P"]).cuda()
    v0 = torch.from_numpy(sc.state["v"]).cuda()
    E = torch.from_numpy(sc.extra["E"]).cuda()
    fwd_ms, bwd_ms = [], []
    with torch.cuda.stream(side):
        for it in range(warmup + steps):
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            ev[0].record(side)
            loss = roll.forward(x0, v0, E, sc.extra["target"])
            ev[1].record(side)
            roll.backward(1.0)
            ev[2].record(side)
            torch.cuda.synchronize()
            if it >= warmup:
                fwd_ms.append(ev[0].elapsed_time(ev[1]))
                bwd_ms.append(ev[1].elapsed_time(ev[2]))
    events = roll.events()
    launches = roll.launches()
    roll.cleanup()
    eng = engine_for_scene(sc)
    eng.numSubsteps = sc.substeps
    eng.step(sc.params.dt * sc.substeps, side)
    eng.sync()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(side)
    for _ in range(steps):
        eng.step(sc.params.dt * sc.substeps, side)
    e1.record(side)
    torch.cuda.synchronize()
    eng_ms = e0.elapsed_time(e1) / steps
    eng.cleanup()
    f, b = float(np.median(fwd_ms)), float(np.median(bwd_ms))
    return {"workload": sc.name, "particles": sc.n, "grid": list(sc.params.grid_res), "substeps": sc.substeps,
            "checkpoint_every": sc.extra["checkpoint_every"], "forward_ms": f, "backward_ms": b, "ratio_backward_to_forward": b / f,
            "ratio_backward_to_engine_forward": b / eng_ms, "engine_forward_ms": eng_ms, "loss": float(loss), "events": events,
            "steps": steps, "warmup": warmup, "launches_total": launches,
            "note": "forward = rollout with checkpoint copies; backward = segment recomputation + reverse G2P/grid/P2G; "
                    "engine_forward = the brick-sparse engine advancing the same scene (uniform E) for the same substeps"}


def measure_mesh_sdf(cpu: bool) -> dict:
    """The collider SDF built from a triangle mesh on the GPU (the reference's
    buildMeshSDF): a 20,480-triangle sphere into the 256^3 grid of the slope
    workload and into a 128^3 grid, timed by CUDA events (median of 3 after
    one untimed), through the prepared mesh the engine's setColliderMesh /
    setColliderMeshPose use (nebula_mpm_mesh_build_sdf: clustered) and through
    the one-shot call on a device list (nebula_mpm_mesh_sdf); with `cpu`, the
    CPU oracle (brute force over cells x triangles, OpenMP) on a 1,280-triangle
    sphere at 48^3 beside the GPU build of the same case."""
    import ctypes as C

    import torch

    from nebula_b200 import _capi, mesh
    from nebula_b200 import scenes as S

    def gpu_ms(tris, res, prepared):
        total = S.hash_cells((res, res, res))
        out = torch.empty(total, dtype=torch.float32, device="cuda")
        r = (C.c_uint32 * 3)(res, res, res)
        s = torch.cuda.current_stream()
        t = torch.from_numpy(tris).cuda()
        m = C.c_void_p()
        if prepared:
            _capi.call("nebula_mpm_mesh_create", tris.ctypes.data_as(C.c_void_p), tris.shape[0], C.byref(m))
        ms = []
        try:
            for it in range(4):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(s)
                if prepared:
                    _capi.call("nebula_mpm_mesh_build_sdf", m, None, None, r, total, C.c_float(1.0 / res), C.c_void_p(out.data_ptr()),
                               C.c_void_p(s.cuda_stream))
                else:
                    _capi.call("nebula_mpm_mesh_sdf", C.c_void_p(t.data_ptr()), tris.shape[0], r, total, C.c_float(1.0 / res),
                               C.c_void_p(out.data_ptr()), C.c_void_p(s.cuda_stream))
                e1.record(s)
                torch.cuda.synchronize()
                if it:
                    ms.append(e0.elapsed_time(e1))
        finally:
            if prepared:
                _capi.call("nebula_mpm_mesh_destroy", m)
        return float(np.median(ms)), out

    res = {}
    big = mesh.icosphere((0.5, 0.5, 0.5), 0.3, 5)
    for n in (256, 128):
        for prepared, tag in ((True, "prepared"), (False, "one_shot")):
            ms, _ = gpu_ms(big, n, prepared)
            res["%s_ms_%d" % (tag, n)] = ms
            res["%s_cell_triangle_pairs_per_s_%d" % (tag, n)] = n ** 3 * big.shape[0] / (ms * 1e-3)
    res["triangles"] = int(big.shape[0])
    if cpu:
        import oracle
        small = mesh.icosphere((0.5, 0.5, 0.5), 0.3, 3)
        g, out = gpu_ms(small, 48, True)
        t0 = time.perf_counter()
        ref = oracle.mesh_sdf(small, (48, 48, 48), S.hash_cells((48, 48, 48)), 1.0 / 48)
        cms = (time.perf_counter() - t0) * 1e3
        res["sample"] = {"triangles": int(small.shape[0]), "grid": 48, "gpu_ms": g, "cpu_ms": cms, "cpu_cores": oracle.num_threads(),
                         "max_abs_diff": float(np.abs(out.cpu().numpy() - ref).max())}
    return res


def measure_pbf_hash(cpu: bool) -> dict:
    """The PBF engine's spatial hash on the shared counting sort
    (nebula_hash_bin): the default FluidEngine buffer (160,592 slots, 30,000 of
    them unused, 64^3 cells; L2-resident and launch-bound) and 8,388,608
    uniform particles on 128^3 cells (160 MB of inputs, larger than L2), timed
    by CUDA events (median of 20 after 3 untimed).  Algorithmic bytes per build: 20 per slot
    (predP + typeFlag read), 4 per included particle (sortedIdx), 12 per cell
    (cellCount zeroed and written, cellOffset written)."""
    import torch

    from nebula_b200 import hash as H

    def timed(grid, p, f):
        hs = H.SpatialHash(grid, len(p))
        pt = torch.from_numpy(p).cuda()
        ft = torch.from_numpy(f.view(np.int32)).cuda()
        s = torch.cuda.current_stream()
        ms = []
        for it in range(23):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            hs.build(pt, ft, s)
            e1.record(s)
            torch.cuda.synchronize()
            if it >= 3:
                ms.append(e0.elapsed_time(e1))
        t = float(np.median(ms))
        m = int((f != H.TYPE_FLAG_UNUSED).sum())
        byts = 20.0 * len(p) + 4.0 * m + 12.0 * grid.hash_cells
        return {"slots": len(p), "included": m, "hash_cells": grid.hash_cells, "ms": t, "particles_per_s": len(p) / (t * 1e-3),
                "algorithmic_bytes": byts, "gbs": byts / (t * 1e-3) / 1e9}

    out = {}
    p, f = H.fluid_layout()
    out["fluid_default"] = timed(H.FluidGrid(), p, f)
    rng = np.random.default_rng(12)
    n = 1 << 23
    q = np.zeros((n, 4), np.float32)
    q[:, :3] = rng.uniform(0.0, 20.0, (n, 3)).astype(np.float32)
    fq = np.zeros(n, np.uint32)
    out["uniform_8m_128"] = timed(H.FluidGrid(cell_size=20.0 / 128.0), q, fq)
    out["uniform_8m_128"]["hbm_frac_of_measured"] = out["uniform_8m_128"]["gbs"] / peaks()[0]
    if cpu:
        import oracle
        g = H.FluidGrid()
        t0 = time.perf_counter()
        for _ in range(5):
            oracle.hash_bin(p, f, g.world_min, g.cell_size, g.grid_res, g.hash_cells)
        out["cpu_fluid_default_ms"] = (time.perf_counter() - t0) * 1e3 / 5
        out["cpu_note"] = "CPU oracle, one thread, same buffer"
    return out


def timed_steps(run_step, steps, stream, flush=None):
    """Device time (ms, CUDA events on `stream`) of `steps` calls of run_step.
    With `flush` (a device buffer larger than L2) the buffer is rewritten
    before every step, outside the events, and the per-step times are summed."""
    import torch
    if flush is None:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            run_step()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)
    evs = []
    for k in range(steps):
        with torch.cuda.stream(stream):
            flush.fill_(float(k & 1))
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        run_step()
        b.record(stream)
        evs.append((a, b))
    torch.cuda.synchronize()
    return sum(a.elapsed_time(b) for a, b in evs)


# ----------------------------------------------------------------------------- nebula arm
def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))

    from nebula_b200 import build as nbuild
    if rank == 0 or world == 1:
        nbuild.build()
    if dist:
        dist.barrier()
    if args.mesh_sdf_only:
        if rank == 0:
            print(json.dumps({"mesh_sdf": measure_mesh_sdf(world == 1 and not args.no_cpu_baseline),
                              "pbf_hash": measure_pbf_hash(world == 1 and not args.no_cpu_baseline)}), flush=True)
        if dist:
            dist.destroy_process_group()
        return
    from nebula_b200.engine import engine_for_scene

    sc = make_scene(args.workload)
    sp = sc.params
    n = sc.n
    S = args.substeps
    eng = engine_for_scene(sc, pipeline=args.pipeline)
    eng.numSubsteps = S
    stream = torch.cuda.current_stream()
    dt_frame = sp.dt * S

    # active nodes A (nodes with mass >= 1e-10 after P2G of the initial state)
    mom, mass = eng.export_grid(sp.dt)
    active = int((mass >= 1e-10).sum())
    del mom, mass

    # ---- launch shape: the autotuner's pick for this GPU and workload (timed outside the bench region)
    tuned = None
    if not args.no_tune and args.pipeline == "fused":
        from nebula_b200 import autotune
        shape, rep = autotune.tune_engine(eng, sc, substeps=S)
        tuned = {"shape": rep["shape"], "source": rep["source"], "ms_per_substep": rep["ms_per_substep"],
                 "default_ms_per_substep": rep["default_ms_per_substep"], "shapes_tried": len(rep["tried"]), "key": rep["key"]}

    # warm-up steps from the initial state, then the initial state again: the
    # timed steps cover substeps 1 .. steps * substeps of the workload
    for _ in range(args.warmup):
        eng.step(dt_frame, stream)
    eng.sync()
    eng.upload_state(sc.state)
    eng.sync()

    # ---- L2: inputs larger than L2, or a flush written between the timed steps
    l2 = torch.cuda.get_device_properties(local).L2_cache_size
    working = 2 * n * 128 + sp.hash_cells * 16 * 3  # both state buffers (8 float4 per particle) + grid acc/vel/vold
    flush = None if working > l2 else torch.empty(2 * l2 // 4, dtype=torch.float32, device="cuda")
    if flush is None:
        l2_note = "inputs larger than L2 (%.0f MB particle state + %d-cell grid, %.0f MB L2)" % (2 * n * 128 / 1e6, sp.hash_cells, l2 / 1e6)
    else:
        l2_note = ("L2 flushed between timed steps (%.0f MB written outside the timed events; working set %.1f MB, %.0f MB L2)"
                   % (flush.numel() * 4 / 1e6, working / 1e6, l2 / 1e6))

    # ---- device-timed region
    st0 = eng.stats()
    clocks = ClockSampler(local)
    clocks.start()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ms = timed_steps(lambda: eng.step(dt_frame, stream), args.steps, stream, flush)
    if dist:
        dist.barrier()
    ck = clocks.stop()
    eng.sync()
    st1 = eng.stats()
    launches = int(st1["kernel_launches"] - st0["kernel_launches"])
    # per-phase split: the same warm-up and steps replayed from the initial state with events
    # between the phases (the work per substep grows as the slab settles, so the window must match)
    prof_steps = args.steps
    eng.upload_state(sc.state)
    for _ in range(args.warmup):
        eng.step(dt_frame, stream)
    eng.sync()
    eng.upload_state(sc.state)
    eng.sync()
    eng.profile(True)
    eng.profile_read(reset=True)
    for _ in range(prof_steps):
        eng.step(dt_frame, stream)
    eng.sync()
    phases = eng.profile_read(reset=True)
    eng.profile(False)
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    total_ps = float(n) * S * args.steps * world
    value = total_ps / (ms * 1e-3)

    # ---- end to end through the C ABI with host buffers (pinned)
    pinned = {f: torch.empty((n, 4), dtype=torch.float32, pin_memory=True) for f in sc.state}
    for f, a in sc.state.items():
        pinned[f].copy_(torch.from_numpy(a))
    host_state = {f: t.numpy() for f, t in pinned.items()}
    out = {f: torch.empty((n, 4), dtype=torch.float32, pin_memory=True).numpy() for f in sc.state}
    from nebula_b200 import _capi
    import ctypes as C
    from nebula_b200.scenes import FIELDS as STATE_FIELDS
    out_ptrs = (C.c_void_p * 8)(*[out[f].ctypes.data for f in STATE_FIELDS])
    e2e_steps = max(2, min(args.steps, 20))
    eng.sync()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()

    in_ptrs = (C.c_void_p * 8)(*[host_state[f].ctypes.data for f in STATE_FIELDS])
    h = C.c_void_p(stream.cuda_stream or None)
    if flush is None:
        # streamed: step k's result goes to the host and step k + 1's input to
        # the device on the engine's copy streams while step k computes
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        _capi.call("nebula_mpm_upload_state_async", eng._h, in_ptrs, n, h)
        for k in range(e2e_steps):
            eng.step(dt_frame, stream)
            _capi.call("nebula_mpm_download_state_async", eng._h, out_ptrs, 4 * n, h)
            if k + 1 < e2e_steps:
                _capi.call("nebula_mpm_upload_state_async", eng._h, in_ptrs, n, h)
        _capi.call("nebula_mpm_wait_downloads", eng._h, h)
        e1.record(stream)
        torch.cuda.synchronize()
        eng.sync()
        ms_e2e = e0.elapsed_time(e1)
        e2e_mode = "streamed: nebula_mpm_upload_state_async / step / nebula_mpm_download_state_async, copies overlapped with the previous step"
    else:
        def e2e_step():
            eng.upload_state(host_state)
            eng.step(dt_frame, stream)
            _capi.call("nebula_mpm_download_state", eng._h, out_ptrs, 4 * n)

        ms_e2e = timed_steps(e2e_step, e2e_steps, stream, flush)
        e2e_mode = "synchronous per step: nebula_mpm_upload_state / step / nebula_mpm_download_state (L2 flushed between steps)"
    if dist:
        t = torch.tensor([ms_e2e], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_e2e = float(t.item())
    e2e_value = float(n) * S * e2e_steps * world / (ms_e2e * 1e-3)
    state_bytes = n * 16 * 8

    # ---- roofline of the dominant phase
    hbm, src = peaks()
    flip = sp.flip_ratio > 0.01
    sdf = sc.sdf is not None
    dom = max((p for p in phases if phases[p][1] > 0), key=lambda p: phases[p][0])
    dom_ms, dom_launches = phases[dom]
    calls = prof_steps * S
    per_launch_ms = dom_ms / calls
    alg = algorithmic_bytes(dom, n, active, sp.hash_cells, flip, sdf)
    achieved = alg / (per_launch_ms * 1e-3) / 1e9
    # dram__bytes_read.sum + dram__bytes_write.sum of one launch, from the committed ncu summary
    traffic = None
    tf = ROOT / "profiles" / ("%s_%s.txt" % (dom, sc.name.replace("slope_flow", "slope")))
    if tf.exists():
        for ln in tf.read_text().splitlines():
            if ln.startswith("dram_bytes_per_launch"):
                traffic = float(ln.split("=")[1])
    roofline = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm, "traffic": traffic,
                "kernel": dom, "algorithmic_bytes_per_launch": alg, "ms_per_launch": per_launch_ms, "peak_source": src + " (hbm_gbs)"}
    substep_ms = ms / (args.steps * S)
    canon = canonical_bytes(n, active, flip, sdf)

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded)",
        "config": {"workload": sc.name, "particles": n, "grid": list(sp.grid_res), "substeps_per_step": S, "dt": sp.dt,
                   "substep_range": [1, args.steps * S], "workload_substeps": sc.substeps,
                   "transfer": "APIC" if sp.flip_ratio < -0.5 else ("FLIP" if flip else "PIC"), "parallelism": "replicas" if world > 1 else "single", "pipeline": args.pipeline,
                   "l2": l2_note, "active_nodes": active},
        "roofline": roofline,
        "substep": {"ms": substep_ms, "canonical_bytes": canon, "canonical_frac": canon / (substep_ms * 1e-3) / 1e9 / hbm,
                    "phases_ms_per_substep": {p: v[0] / calls for p, v in phases.items() if v[1] > 0}},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": state_bytes, "d2h_bytes_per_step": state_bytes,
                "steps": e2e_steps, "mode": e2e_mode},
        "gpu_launches": launches,
        "clocks": ck,
        "autotune": tuned,
    }

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        o, kind, cores, what = cpu_reference(sc)
        k = args.cpu_sample_substeps or 0
        t0 = time.perf_counter()
        o.substep()
        one = time.perf_counter() - t0
        if k == 0:
            k = max(1, min(30, int(15.0 / max(one, 1e-3))))
        t0 = time.perf_counter()
        o.run(k)
        cdt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": n * k / cdt, "unit": UNIT, "cores": cores, "kind": kind,
                                "sample": "%d substeps of %s (after one untimed), %s" % (k, sc.name, what)}
    eng.cleanup()
    if not args.no_batch:
        line["batched"] = measure_batch(args.batch_steps, max(1, min(args.warmup, 3)), 20, dist, tune=not args.no_tune)
    if not args.no_adjoint:
        line["adjoint"] = measure_adjoint(3, 2)
    if not args.no_mesh_sdf:
        line["mesh_sdf"] = measure_mesh_sdf(rank == 0 and world == 1 and not args.no_cpu_baseline)
        line["pbf_hash"] = measure_pbf_hash(rank == 0 and world == 1 and not args.no_cpu_baseline)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
