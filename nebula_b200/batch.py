"""Python binding of ``nebula::BatchEngine`` (the ``nebula_mpm_batch_*`` C ABI).

A batch holds many independent scenes with the single-scene engine's
parameter surface and advances all of them with one set of launches per
substep (one brick space, one particle array, a CUDA graph per step).  The
reference has no batched form; per scene the physics is the plain engine's.

    b = BatchEngine(max_scenes=64, max_particles=3_000_000)
    ids = [b.add_scene_from(sc) for sc in scenes]
    b.set_collider_track(ids[0], track)      # (substeps, colliders) records
    b.step(dt * 200, 200, stream=torch.cuda.current_stream())
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi
from ._capi import call
from .engine import FIELD_INDEX, MPMConfig, _PARAM_NAMES, _ptr, _stream_handle
from .scenes import COLLIDER_DTYPE, FIELDS, FORCE_DTYPE, MATERIAL_DTYPE


class BatchEngine:
    def __init__(self, max_scenes: int, max_particles: int):
        cfg = _capi.BatchConfig(int(max_scenes), int(max_particles))
        h = C.c_void_p()
        call("nebula_mpm_batch_create", C.byref(cfg), C.byref(h))
        self._h = h

    def cleanup(self):
        if getattr(self, "_h", None) and self._h.value:
            call("nebula_mpm_batch_destroy", self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.cleanup()
        except Exception:
            pass

    # ------------------------------------------------------------ scenes
    def add_scene(self, cfg: MPMConfig, pos4, vel4) -> int:
        p = np.ascontiguousarray(pos4, dtype=np.float32).reshape(-1, 4)
        v = np.ascontiguousarray(vel4, dtype=np.float32).reshape(-1, 4)
        if p.shape != v.shape:
            raise ValueError("pos and vel must have the same shape")
        s = C.c_uint32()
        call("nebula_mpm_batch_add_scene", self._h, C.byref(cfg.to_c()), _ptr(p), _ptr(v), p.shape[0], C.byref(s))
        return s.value

    def add_scene_from(self, scene) -> int:
        """Add a ``scenes.Scene`` (domain, transfer mode, materials, forces,
        colliders, SDF) and upload its full particle state."""
        sp = scene.params
        cfg = MPMConfig(nx=0, ny=0, nz=0, domainSize=tuple(sp.domain_size), cellSize=sp.cell_size, maxParticles=0, E=1e4, nu=0.3,
                        rho0=sp.rho0)
        s = self.add_scene(cfg, scene.state["P"], scene.state["v"])
        self.set_params(s, flip_ratio=sp.flip_ratio, M_friction=sp.M_friction, q_cohesion=sp.q_cohesion, q_max=sp.q_max,
                        plasticModel=sp.plastic_model)
        if sp.materials:
            self.set_materials(s, sp.materials_array()[: len(sp.materials)])
        if sp.forces:
            self.set_forces(s, list(sp.forces))
        if sp.colliders:
            self.set_colliders(s, sp.colliders_array()[: len(sp.colliders)])
        if scene.sdf is not None:
            self.set_collider_sdf(s, scene.sdf)
        self.upload_state(s, scene.state)
        return s

    def params(self, s: int) -> dict:
        p = _capi.Params()
        call("nebula_mpm_batch_get_params", self._h, s, C.byref(p))
        return {k: getattr(p, k) for k in _PARAM_NAMES}

    def set_params(self, s: int, **kw):
        p = _capi.Params()
        call("nebula_mpm_batch_get_params", self._h, s, C.byref(p))
        for k, v in kw.items():
            if k not in _PARAM_NAMES:
                raise KeyError(k)
            setattr(p, k, v)
        call("nebula_mpm_batch_set_params", self._h, s, C.byref(p))

    def set_materials(self, s: int, mats):
        a = np.ascontiguousarray(np.asarray(mats, dtype=MATERIAL_DTYPE).reshape(-1))
        call("nebula_mpm_batch_set_materials", self._h, s, _ptr(a), len(a))

    def set_particle_material_ids(self, s: int, ids):
        a = np.ascontiguousarray(ids, dtype=np.uint32)
        call("nebula_mpm_batch_set_particle_material_ids", self._h, s, _ptr(a), len(a))

    def set_colliders(self, s: int, cols):
        a = np.ascontiguousarray(np.asarray(cols, dtype=COLLIDER_DTYPE).reshape(-1))
        call("nebula_mpm_batch_set_colliders", self._h, s, _ptr(a), len(a))

    def set_collider_track(self, s: int, track):
        a = np.ascontiguousarray(np.asarray(track, dtype=COLLIDER_DTYPE))
        if a.ndim == 1:
            a = a.reshape(-1, 1)
        call("nebula_mpm_batch_set_collider_track", self._h, s, _ptr(a), a.shape[1], a.shape[0])

    def set_collider_sdf(self, s: int, morton_sdf):
        a = np.ascontiguousarray(morton_sdf, dtype=np.float32)
        call("nebula_mpm_batch_set_collider_sdf", self._h, s, _ptr(a), a.size)

    def clear_collider_sdf(self, s: int):
        call("nebula_mpm_batch_clear_collider_sdf", self._h, s)

    def set_forces(self, s: int, forces):
        a = np.zeros(max(1, len(forces)), FORCE_DTYPE)
        for i, f in enumerate(forces):
            a[i] = f
        call("nebula_mpm_batch_set_forces", self._h, s, _ptr(a), len(forces))

    # ------------------------------------------------------------ particles
    def scene_info(self, s: int) -> dict:
        i = _capi.SceneInfo()
        call("nebula_mpm_batch_scene_info", self._h, s, C.byref(i))
        return {k: (list(getattr(i, k)) if k == "grid_res" else getattr(i, k)) for k, _ in i._fields_}

    def upload_state(self, s: int, state: dict):
        arrs = [np.ascontiguousarray(state[f], dtype=np.float32).reshape(-1, 4) for f in FIELDS]
        ptrs = (C.c_void_p * 8)(*[a.ctypes.data for a in arrs])
        call("nebula_mpm_batch_upload_state", self._h, s, ptrs, arrs[0].shape[0])

    def download(self, s: int, field: str) -> np.ndarray:
        n = self.scene_info(s)["particles"]
        out = np.empty((n, 4), np.float32)
        call("nebula_mpm_batch_download", self._h, s, FIELD_INDEX[field], _ptr(out), out.size)
        return out

    def state(self, s: int) -> dict:
        return {f: self.download(s, f) for f in FIELDS}

    # ------------------------------------------------------------ stepping
    def step(self, dt: float, substeps: int, stream=None):
        """`substeps` substeps of dt/substeps for every scene, on `stream`."""
        call("nebula_mpm_batch_step", self._h, float(dt), int(substeps), _stream_handle(stream))

    def run_substeps(self, sub_dt: float, count: int, stream=None):
        self.step(sub_dt * count, count, stream)

    def set_launch_config(self, cfg):
        """Launch shape of the fused and grid kernels (autotune.LaunchShape or a
        dict with its fields); drops the batch's captured graphs."""
        from .autotune import LaunchShape
        c = LaunchShape.coerce(cfg).to_c()
        call("nebula_mpm_batch_set_launch_config", self._h, C.byref(c))

    def launch_config(self):
        from .autotune import LaunchShape
        c = _capi.LaunchConfig()
        call("nebula_mpm_batch_get_launch_config", self._h, C.byref(c))
        return LaunchShape.from_c(c)

    def set_graphs(self, enable: bool):
        call("nebula_mpm_batch_set_graphs", self._h, int(bool(enable)))

    def sync(self):
        call("nebula_mpm_batch_sync", self._h)

    def stats(self) -> dict:
        s = _capi.BatchStats()
        call("nebula_mpm_batch_get_stats", self._h, C.byref(s))
        return {k: getattr(s, k) for k, _ in s._fields_}


def batch_for_scenes(scenes, capacity: int | None = None) -> tuple[BatchEngine, list[int]]:
    """A batch holding every scene of `scenes` (in order)."""
    total = sum(sc.n for sc in scenes)
    b = BatchEngine(max(1, len(scenes)), int(capacity or total))
    return b, [b.add_scene_from(sc) for sc in scenes]
