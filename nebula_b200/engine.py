"""Python binding of the C++ ``nebula::MPMEngine`` (include/nebula_mpm.h).

Method names follow the reference's ``MPMEngine`` (src/engine/MPMEngine.h:59-186)
and ``EngineBase`` force API (src/engine/EngineBase.h:27-31), so code written
against the reference reads the same:

    eng = MPMEngine(MPMConfig(nx=20, ny=20, nz=20, domainSize=(1,1,1), cellSize=1/64))
    eng.flip_ratio = -1.0
    eng.addForce(gravity())
    eng.step(dt)

Everything runs in the CUDA library; this module only marshals arguments.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _capi
from ._capi import call
from .scenes import COLLIDER_DTYPE, EMITTER_DTYPE, FIELDS, FORCE_DTYPE, MATERIAL_DTYPE

FIELD_INDEX = {f: i for i, f in enumerate(FIELDS)}


@dataclass
class MPMConfig:
    """MPMConfig (src/engine/MPMEngine.h:22-55)."""
    nx: int = 32
    ny: int = 32
    nz: int = 32
    domainSize: tuple = (10.0, 10.0, 10.0)
    cellSize: float = 10.0 / 64.0
    maxParticles: int = 0
    E: float = 1e4
    nu: float = 0.3
    rho0: float = 1000.0

    def to_c(self) -> _capi.Config:
        c = _capi.Config()
        c.nx, c.ny, c.nz = self.nx, self.ny, self.nz
        c.domainSize[:] = [float(v) for v in self.domainSize]
        c.cellSize = self.cellSize
        c.maxParticles = self.maxParticles
        c.E, c.nu, c.rho0 = self.E, self.nu, self.rho0
        return c


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def _stream_handle(stream):
    if stream is None:
        return None
    if isinstance(stream, int):
        return C.c_void_p(stream)
    h = getattr(stream, "cuda_stream", None)  # torch.cuda.Stream
    return C.c_void_p(h) if h else None


_PARAM_NAMES = ("restitution", "wall_friction", "numSubsteps", "plasticModel", "q_max", "M_friction", "q_cohesion", "flip_ratio")



def lattice_record(counts, spacing, origin, jitter, seed, stream=0, particle_volume=0.0, vel=(0.0, 0.0, 0.0), material_id=0):
    """A nebula_mpm_lattice: the seeded jittered lattice of scenes.jittered_lattice."""
    L = _capi.Lattice()
    L.counts[:] = [int(c) for c in counts]
    L.materialId = int(material_id)
    L.spacing = float(spacing)
    L.origin[:] = [float(o) for o in origin]
    L.jitter = float(jitter)
    L.seed = int(seed)
    L.stream = int(stream)
    L.particleVolume = float(particle_volume)
    L.vel[:] = [float(v) for v in vel]
    return L


def lattice_points(L) -> tuple[np.ndarray, np.ndarray]:
    """(pos4, vel4) of a lattice record, computed on the host by the library."""
    n = int(L.counts[0]) * int(L.counts[1]) * int(L.counts[2])
    pos = np.empty((n, 4), np.float32)
    vel = np.empty((n, 4), np.float32)
    call("nebula_mpm_lattice_points", C.byref(L), _ptr(pos), _ptr(vel), n)
    return pos, vel

class MPMEngine:
    """One MPM scene on the GPU."""

    def __init__(self, cfg: MPMConfig | None = None):
        cfg = cfg or MPMConfig()
        self.cfg = cfg
        h = C.c_void_p()
        call("nebula_mpm_create", C.byref(cfg.to_c()), C.byref(h))
        self._h = h
        self._forces = []

    # ------------------------------------------------------------ lifetime
    def cleanup(self):
        if getattr(self, "_h", None) and self._h.value:
            call("nebula_mpm_destroy", self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.cleanup()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.cleanup()

    # ------------------------------------------------------------ public fields (MPMEngine.h:72-80)
    def _params(self) -> _capi.Params:
        p = _capi.Params()
        call("nebula_mpm_get_params", self._h, C.byref(p))
        return p

    def __getattr__(self, name):
        if name in _PARAM_NAMES:
            return getattr(self._params(), name)
        raise AttributeError(name)

    def __setattr__(self, name, value):
        if name in _PARAM_NAMES:
            p = self._params()
            setattr(p, name, value)
            call("nebula_mpm_set_params", self._h, C.byref(p))
        else:
            object.__setattr__(self, name, value)

    # ------------------------------------------------------------ tables
    def setMaterials(self, mats):
        a = np.ascontiguousarray(np.asarray(mats, dtype=MATERIAL_DTYPE).reshape(-1))
        call("nebula_mpm_set_materials", self._h, _ptr(a), len(a))

    def setParticleMaterialIds(self, ids):
        a = np.ascontiguousarray(ids, dtype=np.uint32)
        call("nebula_mpm_set_particle_material_ids", self._h, _ptr(a), len(a))

    def setColliders(self, cols):
        a = np.ascontiguousarray(np.asarray(cols, dtype=COLLIDER_DTYPE).reshape(-1))
        call("nebula_mpm_set_colliders", self._h, _ptr(a), len(a))

    def setColliderTrack(self, track):
        """track: (substeps, perSubstep) collider records; substep k of each
        later step uses set min(k, substeps - 1)."""
        a = np.ascontiguousarray(np.asarray(track, dtype=COLLIDER_DTYPE))
        if a.ndim == 1:
            a = a.reshape(-1, 1)
        call("nebula_mpm_set_collider_track", self._h, _ptr(a), a.shape[1], a.shape[0])

    def clearAnalyticColliders(self):
        call("nebula_mpm_clear_analytic_colliders", self._h)

    def setColliderSDF(self, morton_sdf):
        a = np.ascontiguousarray(morton_sdf, dtype=np.float32)
        call("nebula_mpm_set_collider_sdf", self._h, _ptr(a), a.size)

    def setColliderSphere(self, radius, cx, cy, cz):
        call("nebula_mpm_set_collider_sphere", self._h, radius, cx, cy, cz)

    def clearCollider(self):
        call("nebula_mpm_clear_collider", self._h)

    def setColliderMesh(self, tris):
        """setColliderSDF(buildMeshSDF(tris, ...)) with the SDF built on the GPU; tris (n, 12)."""
        a = np.ascontiguousarray(tris, dtype=np.float32).reshape(-1, 12)
        call("nebula_mpm_set_collider_mesh", self._h, _ptr(a), a.shape[0])

    def setColliderMeshPose(self, translation, rotation=(1.0, 0.0, 0.0, 0.0)):
        """setColliderSDF(buildMeshSDF(transformTriangles(tris, translation,
        rotation))) for the triangles of the last setColliderMesh, on the
        device; rotation is a unit quaternion (w, x, y, z)."""
        t = np.ascontiguousarray(translation, dtype=np.float32).reshape(3)
        q = np.ascontiguousarray(rotation, dtype=np.float32).reshape(4)
        call("nebula_mpm_set_collider_mesh_pose", self._h, _ptr(t), _ptr(q))

    def setColliderMeshClosestPoint(self, reference: bool):
        """True: later setColliderMesh / setColliderMeshPose builds take the
        reference's closestPtOnTriangle (no edge-BC region, brute force), so
        the SDF equals the reference's buildMeshSDF output; False (default):
        the complete region test."""
        mode = _capi.CLOSEST_POINT_REFERENCE if reference else _capi.CLOSEST_POINT_COMPLETE
        call("nebula_mpm_set_collider_mesh_closest_point", self._h, mode)

    def setForces(self, forces):
        self._forces = list(forces)
        a = np.zeros(max(1, len(self._forces)), FORCE_DTYPE)
        for i, f in enumerate(self._forces):
            a[i] = f
        call("nebula_mpm_set_forces", self._h, _ptr(a), len(self._forces))

    def addForce(self, f):
        self.setForces(self._forces + [f])

    def removeForce(self, index: int):
        fs = list(self._forces)
        del fs[index]
        self.setForces(fs)

    def clearForces(self):
        self.setForces([])

    # ------------------------------------------------------------ particles
    def appendParticles(self, pos4, vel4) -> int:
        p = np.ascontiguousarray(pos4, dtype=np.float32).reshape(-1, 4)
        v = np.ascontiguousarray(vel4, dtype=np.float32).reshape(-1, 4)
        if p.shape != v.shape:
            raise ValueError("pos and vel must have the same shape")
        k = C.c_uint32()
        call("nebula_mpm_append_particles", self._h, _ptr(p), _ptr(v), p.shape[0], C.byref(k))
        return k.value

    def append_lattice(self, L) -> int:
        """nebula_mpm_append_lattice: the seeded lattice record `L` appended."""
        k = C.c_uint32()
        call("nebula_mpm_append_lattice", self._h, C.byref(L), C.byref(k))
        return k.value

    def resetParticles(self):
        call("nebula_mpm_reset_particles", self._h)

    # ------------------------------------------------------------ emitters (MPMEngine.h:100-104)
    def addEmitter(self, em) -> int:
        a = np.ascontiguousarray(np.asarray(em, dtype=EMITTER_DTYPE).reshape(-1)[:1])
        k = C.c_uint32()
        call("nebula_mpm_add_emitter", self._h, _ptr(a), C.byref(k))
        return k.value

    def clearEmitters(self):
        call("nebula_mpm_clear_emitters", self._h)

    def getEmitter(self, index: int):
        """(record, times emitted)."""
        a = np.zeros(1, EMITTER_DTYPE)
        d = C.c_int32()
        call("nebula_mpm_get_emitter", self._h, index, _ptr(a), C.byref(d))
        return a[0], d.value

    def upload_state(self, state: dict):
        arrs = [np.ascontiguousarray(state[f], dtype=np.float32).reshape(-1, 4) for f in FIELDS]
        n = arrs[0].shape[0]
        ptrs = (C.c_void_p * 8)(*[a.ctypes.data for a in arrs])
        call("nebula_mpm_upload_state", self._h, ptrs, n)

    def upload_state_async(self, state: dict, stream=None):
        """nebula_mpm_upload_state_async: `state` holds 8 C-contiguous (n, 4)
        float32 arrays (pinned host memory for an asynchronous copy), which the
        caller keeps unchanged until `stream` has passed this point."""
        arrs = [state[f] for f in FIELDS]
        for a in arrs:
            if a.dtype != np.float32 or not a.flags.c_contiguous or a.ndim != 2 or a.shape[1] != 4:
                raise ValueError("upload_state_async wants C-contiguous (n, 4) float32 arrays")
        ptrs = (C.c_void_p * 8)(*[a.ctypes.data for a in arrs])
        call("nebula_mpm_upload_state_async", self._h, ptrs, arrs[0].shape[0], _stream_handle(stream))

    def download_state_async(self, out: dict, stream=None):
        """nebula_mpm_download_state_async into 8 C-contiguous (live, 4) float32
        arrays, valid after sync() or once `stream` passed wait_downloads()."""
        arrs = [out[f] for f in FIELDS]
        n = self.liveParticleCount()
        for a in arrs:
            if a.dtype != np.float32 or not a.flags.c_contiguous or a.shape != (n, 4):
                raise ValueError("download_state_async wants C-contiguous (live, 4) float32 arrays")
        ptrs = (C.c_void_p * 8)(*[a.ctypes.data for a in arrs])
        call("nebula_mpm_download_state_async", self._h, ptrs, 4 * n, _stream_handle(stream))

    def wait_downloads(self, stream=None):
        call("nebula_mpm_wait_downloads", self._h, _stream_handle(stream))

    def liveParticleCount(self) -> int:
        n = C.c_uint32()
        call("nebula_mpm_live_count", self._h, C.byref(n))
        return n.value

    def download(self, field: str) -> np.ndarray:
        n = self.liveParticleCount()
        out = np.empty((n, 4), np.float32)
        call("nebula_mpm_download", self._h, FIELD_INDEX[field], _ptr(out), out.size)
        return out

    def device_ptr(self, field: str) -> int:
        """Device address of `field` (4 * live floats, original particle order);
        valid until the next step or particle change."""
        p = C.c_void_p()
        call("nebula_mpm_device_ptr", self._h, FIELD_INDEX[field], C.byref(p))
        return int(p.value or 0)

    def setGravity(self, gx: float, gy: float, gz: float):
        """nebula_mpm_set_gravity on the table this binding keeps: every gravity
        entry replaced by one vector (none for (0, 0, 0)), other forces kept."""
        from .scenes import FORCE_GRAVITY, gravity
        fs = [f for f in self._forces if int(f["type"]) != FORCE_GRAVITY]
        if gx or gy or gz:
            fs.append(gravity((gx, gy, gz)))
        self.setForces(fs)

    def state(self) -> dict:
        """All 8 fields (one unpermute, one synchronisation)."""
        n = self.liveParticleCount()
        out = {f: np.empty((n, 4), np.float32) for f in FIELDS}
        ptrs = (C.c_void_p * 8)(*[out[f].ctypes.data for f in FIELDS])
        call("nebula_mpm_download_state", self._h, ptrs, 4 * n)
        return out

    # ------------------------------------------------------------ stepping
    def step(self, dt: float, stream=None):
        """MPMEngine::step: numSubsteps substeps of dt/numSubsteps on `stream`."""
        call("nebula_mpm_step", self._h, float(dt), _stream_handle(stream))

    def run_substeps(self, sub_dt: float, count: int, stream=None):
        """`count` substeps of length sub_dt (one step() call with numSubsteps=count)."""
        old = self.numSubsteps
        self.numSubsteps = int(count)
        try:
            self.step(sub_dt * count, stream)
        finally:
            self.numSubsteps = old

    def sync(self):
        call("nebula_mpm_sync", self._h)

    def stats(self) -> dict:
        s = _capi.Stats()
        call("nebula_mpm_get_stats", self._h, C.byref(s))
        return {k: (list(getattr(s, k)) if k == "grid_res" else getattr(s, k)) for k, _ in s._fields_}

    # ------------------------------------------------------------ pipeline
    def set_graphs(self, enable: bool):
        """Replays of the substep loop from the engine's own CUDA graphs (on by
        default); off drops the captured graphs."""
        call("nebula_mpm_set_graphs", self._h, int(bool(enable)))

    def set_launch_config(self, cfg):
        """Launch shape of the fused and grid kernels (autotune.LaunchShape or a
        dict with its fields)."""
        from .autotune import LaunchShape
        c = LaunchShape.coerce(cfg).to_c()
        call("nebula_mpm_set_launch_config", self._h, C.byref(c))

    def launch_config(self):
        from .autotune import LaunchShape
        c = _capi.LaunchConfig()
        call("nebula_mpm_get_launch_config", self._h, C.byref(c))
        return LaunchShape.from_c(c)

    def set_pipeline(self, name: str):
        """"fused" (default: brick-sparse, fused G2P+P2G) or "dense" (one kernel per reference dispatch)."""
        call("nebula_mpm_set_pipeline", self._h, {"dense": _capi.PIPELINE_DENSE, "fused": _capi.PIPELINE_FUSED}[name])

    def export_brick_bins(self):
        """The engine's brick binning: (brick ids, start slots, original particle id per slot)."""
        st = self.stats()
        nb = max(1, st["hash_cells"] // 64)
        n = st["live_particles"]
        ids = np.empty(nb, np.uint32)
        starts = np.empty(nb + 1, np.uint32)
        pids = np.empty(max(1, n), np.uint32)
        k = C.c_uint32()
        call("nebula_mpm_export_brick_bins", self._h, C.byref(k), _ptr(ids), _ptr(starts), _ptr(pids))
        return ids[: k.value].copy(), starts[: k.value + 1].copy(), pids[:n].copy()

    # ------------------------------------------------------------ device timing
    PHASES = ("bin", "p2g", "grid", "g2p", "g2p2g", "other")

    def profile(self, enable: bool = True):
        call("nebula_mpm_profile_enable", self._h, int(bool(enable)))

    def profile_read(self, reset: bool = True) -> dict:
        ms = np.zeros(6, np.float64)
        ln = np.zeros(6, np.uint64)
        call("nebula_mpm_profile_read", self._h, _ptr(ms), _ptr(ln), int(reset))
        return {p: (float(ms[i]), int(ln[i])) for i, p in enumerate(self.PHASES)}

    # ------------------------------------------------------------ reference-format exports
    def export_bins(self):
        st = self.stats()
        nc, n = st["hash_cells"], st["live_particles"]
        cnt = np.empty(nc, np.uint32)
        off = np.empty(nc, np.uint32)
        srt = np.empty(max(1, n), np.uint32)
        call("nebula_mpm_export_bins", self._h, _ptr(cnt), _ptr(off), _ptr(srt))
        return cnt, off, srt[:n]

    def export_grid(self, dt: float):
        nc = self.stats()["hash_cells"]
        mom = np.empty((nc, 4), np.float32)
        mass = np.empty(nc, np.float32)
        call("nebula_mpm_export_grid", self._h, float(dt), _ptr(mom), _ptr(mass))
        return mom, mass


def engine_for_scene(scene, capacity: int | None = None, pipeline: str = "fused") -> MPMEngine:
    """An engine configured like `scene` (domain, materials, forces, colliders,
    SDF, transfer mode) holding the scene's particle state."""
    sp = scene.params
    cfg = MPMConfig(nx=0, ny=0, nz=0, domainSize=tuple(sp.domain_size), cellSize=sp.cell_size,
                    maxParticles=int(capacity or scene.n), E=1e4, nu=0.3, rho0=sp.rho0)
    eng = MPMEngine(cfg)
    if pipeline != "fused":
        eng.set_pipeline(pipeline)
    eng.flip_ratio = sp.flip_ratio
    eng.M_friction = sp.M_friction
    eng.q_cohesion = sp.q_cohesion
    eng.q_max = sp.q_max
    eng.plasticModel = sp.plastic_model
    if sp.materials:
        eng.setMaterials(sp.materials_array()[: len(sp.materials)])
    if sp.forces:
        eng.setForces(list(sp.forces))
    if sp.colliders:
        eng.setColliders(sp.colliders_array()[: len(sp.colliders)])
    if scene.sdf is not None:
        eng.setColliderSDF(scene.sdf)
    eng.upload_state(scene.state)
    return eng
