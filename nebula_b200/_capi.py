"""ctypes declarations of the C ABI in ``include/nebula_mpm.h``.

Loading fails loudly when ``libnebula_mpm.so`` is missing: there is no CPU
fallback for any call.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libnebula_mpm.so"

OK, ERR_INVALID, ERR_CUDA, ERR_OOM, ERR_DEVICE, ERR_UNSUPPORTED = range(6)
CLOSEST_POINT_COMPLETE, CLOSEST_POINT_REFERENCE = 0, 1
PIPELINE_DENSE, PIPELINE_FUSED = 0, 1


class NebulaError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__("nebula_mpm error %d: %s" % (code, msg))
        self.code = code


class Config(C.Structure):
    _fields_ = [("nx", C.c_uint32), ("ny", C.c_uint32), ("nz", C.c_uint32), ("domainSize", C.c_float * 3),
                ("cellSize", C.c_float), ("maxParticles", C.c_uint32), ("E", C.c_float), ("nu", C.c_float), ("rho0", C.c_float)]


class Params(C.Structure):
    _fields_ = [("restitution", C.c_float), ("wall_friction", C.c_float), ("numSubsteps", C.c_int32), ("plasticModel", C.c_uint32),
                ("q_max", C.c_float), ("M_friction", C.c_float), ("q_cohesion", C.c_float), ("flip_ratio", C.c_float)]


class Lattice(C.Structure):
    _fields_ = [("counts", C.c_uint32 * 3), ("materialId", C.c_uint32), ("spacing", C.c_double), ("origin", C.c_double * 3),
                ("jitter", C.c_double), ("seed", C.c_uint64), ("stream", C.c_uint64), ("particleVolume", C.c_float),
                ("vel", C.c_float * 3)]


class Stats(C.Structure):
    _fields_ = [("substeps", C.c_uint64), ("live_particles", C.c_uint32), ("active_bricks", C.c_uint32), ("particle_bricks", C.c_uint32),
                ("grid_res", C.c_uint32 * 3), ("cube_res", C.c_uint32), ("hash_cells", C.c_uint32), ("kernel_launches", C.c_uint64),
                ("overflow_particles", C.c_uint32), ("error_flags", C.c_uint32), ("graph_launches", C.c_uint64)]


class Pass(C.Structure):
    _fields_ = [("dt", C.c_float), ("cellSize", C.c_float), ("gridRes", C.c_uint32 * 3), ("hashCells", C.c_uint32),
                ("worldMin", C.c_float * 3), ("worldMax", C.c_float * 3), ("flip_ratio", C.c_float), ("particleCount", C.c_uint32),
                ("materialCount", C.c_uint32), ("colliderCount", C.c_uint32), ("forceCount", C.c_uint32), ("mu_lame", C.c_float),
                ("lambda_lame", C.c_float), ("rho0", C.c_float), ("M_friction", C.c_float), ("q_cohesion", C.c_float), ("q_max", C.c_float),
                ("plasticModel", C.c_uint32)]


class Particles(C.Structure):
    _fields_ = [("f", C.c_void_p * 8)]


class LaunchConfig(C.Structure):
    _fields_ = [("fused_threads", C.c_uint32), ("fused_ctas_per_sm", C.c_uint32), ("grid_ctas_per_sm", C.c_uint32), ("grid_batch", C.c_uint32),
                ("fused_split", C.c_uint32)]


class BatchConfig(C.Structure):
    _fields_ = [("maxScenes", C.c_uint32), ("maxParticles", C.c_uint32)]


class SceneInfo(C.Structure):
    _fields_ = [("grid_res", C.c_uint32 * 3), ("cube_res", C.c_uint32), ("hash_cells", C.c_uint32), ("particles", C.c_uint32),
                ("first_brick", C.c_uint32), ("bricks", C.c_uint32)]


class BatchStats(C.Structure):
    _fields_ = [("substeps", C.c_uint64), ("scenes", C.c_uint32), ("live_particles", C.c_uint32), ("total_bricks", C.c_uint32),
                ("active_bricks", C.c_uint32), ("particle_bricks", C.c_uint32), ("overflow_particles", C.c_uint32),
                ("kernel_launches", C.c_uint64), ("graph_launches", C.c_uint64), ("error_flags", C.c_uint32)]


class AdjointConfig(C.Structure):
    _fields_ = [("domainSize", C.c_float * 3), ("cellSize", C.c_float), ("particles", C.c_uint32), ("substeps", C.c_uint32),
                ("checkpointEvery", C.c_uint32), ("dt", C.c_float), ("gravity", C.c_float * 3), ("nu", C.c_float), ("rho0", C.c_float)]


_lib = None

# name -> (restype, argtypes)
_SIGS = {
    "nebula_mpm_create": (C.c_int, [C.POINTER(Config), C.POINTER(C.c_void_p)]),
    "nebula_mpm_destroy": (C.c_int, [C.c_void_p]),
    "nebula_mpm_last_error": (C.c_char_p, []),
    "nebula_mpm_set_params": (C.c_int, [C.c_void_p, C.POINTER(Params)]),
    "nebula_mpm_get_params": (C.c_int, [C.c_void_p, C.POINTER(Params)]),
    "nebula_mpm_set_materials": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32]),
    "nebula_mpm_set_particle_material_ids": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32]),
    "nebula_mpm_set_colliders": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32]),
    "nebula_mpm_clear_analytic_colliders": (C.c_int, [C.c_void_p]),
    "nebula_mpm_set_collider_sdf": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64]),
    "nebula_mpm_set_collider_sphere": (C.c_int, [C.c_void_p, C.c_float, C.c_float, C.c_float, C.c_float]),
    "nebula_mpm_clear_collider": (C.c_int, [C.c_void_p]),
    "nebula_mpm_set_collider_mesh": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32]),
    "nebula_mpm_mesh_sdf": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32 * 3, C.c_uint32, C.c_float, C.c_void_p, C.c_void_p]),
    "nebula_mpm_mesh_create": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p]),
    "nebula_mpm_mesh_destroy": (C.c_int, [C.c_void_p]),
    "nebula_mpm_mesh_build_sdf": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32 * 3, C.c_uint32, C.c_float, C.c_void_p, C.c_void_p]),
    "nebula_mpm_mesh_sdf_posed": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint32 * 3, C.c_uint32, C.c_float,
                                            C.c_void_p, C.c_void_p]),
    "nebula_mpm_set_collider_mesh_pose": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "nebula_mpm_set_collider_mesh_closest_point": (C.c_int, [C.c_void_p, C.c_int]),
    "nebula_mpm_mesh_sdf_reference": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint32 * 3, C.c_uint32, C.c_float,
                                               C.c_void_p, C.c_void_p]),
    "nebula_mpm_mesh_build_sdf_reference": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32 * 3, C.c_uint32, C.c_float, C.c_void_p,
                                                     C.c_void_p]),
    "nebula_mpm_set_forces": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32]),
    "nebula_mpm_append_particles": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.POINTER(C.c_uint32)]),
    "nebula_mpm_reset_particles": (C.c_int, [C.c_void_p]),
    "nebula_mpm_add_emitter": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_uint32)]),
    "nebula_mpm_clear_emitters": (C.c_int, [C.c_void_p]),
    "nebula_mpm_get_emitter": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.POINTER(C.c_int32)]),
    "nebula_mpm_upload_state": (C.c_int, [C.c_void_p, C.c_void_p * 8, C.c_uint32]),
    "nebula_mpm_download": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_uint64]),
    "nebula_mpm_step": (C.c_int, [C.c_void_p, C.c_float, C.c_void_p]),
    "nebula_mpm_live_count": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint32)]),
    "nebula_mpm_get_stats": (C.c_int, [C.c_void_p, C.POINTER(Stats)]),
    "nebula_mpm_sync": (C.c_int, [C.c_void_p]),
    "nebula_mpm_export_bins": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "nebula_mpm_profile_enable": (C.c_int, [C.c_void_p, C.c_int]),
    "nebula_mpm_set_pipeline": (C.c_int, [C.c_void_p, C.c_int]),
    "nebula_mpm_set_launch_config": (C.c_int, [C.c_void_p, C.c_void_p]),
    "nebula_mpm_set_graphs": (C.c_int, [C.c_void_p, C.c_int]),
    "nebula_mpm_download_state": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64]),
    "nebula_mpm_upload_state_async": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]),
    "nebula_mpm_lattice_points": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64]),
    "nebula_mpm_append_lattice": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "nebula_mpm_download_state_async": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p]),
    "nebula_mpm_wait_downloads": (C.c_int, [C.c_void_p, C.c_void_p]),
    "nebula_mpm_device_ptr": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "nebula_mpm_set_gravity": (C.c_int, [C.c_void_p, C.c_float, C.c_float, C.c_float]),
    "nebula_mpm_get_launch_config": (C.c_int, [C.c_void_p, C.c_void_p]),
    "nebula_mpm_launch_limits": (C.c_int, [C.c_int, C.c_int, C.c_void_p, C.c_void_p]),
    "nebula_mpm_probe_wait_expiry": (C.c_int, [C.c_void_p]),
    "nebula_mpm_export_brick_bins": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "nebula_mpm_profile_read": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
    "nebula_mpm_export_grid": (C.c_int, [C.c_void_p, C.c_float, C.c_void_p, C.c_void_p]),
    "nebula_mpm_set_collider_track": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32]),
    "nebula_mpm_batch_create": (C.c_int, [C.POINTER(BatchConfig), C.POINTER(C.c_void_p)]),
    "nebula_mpm_batch_destroy": (C.c_int, [C.c_void_p]),
    "nebula_mpm_batch_add_scene": (C.c_int, [C.c_void_p, C.POINTER(Config), C.c_void_p, C.c_void_p, C.c_uint32, C.POINTER(C.c_uint32)]),
    "nebula_mpm_batch_set_params": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(Params)]),
    "nebula_mpm_batch_get_params": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(Params)]),
    "nebula_mpm_batch_set_materials": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32]),
    "nebula_mpm_batch_set_particle_material_ids": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32]),
    "nebula_mpm_batch_set_colliders": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32]),
    "nebula_mpm_batch_set_collider_track": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_uint32]),
    "nebula_mpm_batch_set_collider_sdf": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint64]),
    "nebula_mpm_batch_clear_collider_sdf": (C.c_int, [C.c_void_p, C.c_uint32]),
    "nebula_mpm_batch_set_forces": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32]),
    "nebula_mpm_batch_upload_state": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p * 8, C.c_uint32]),
    "nebula_mpm_batch_download": (C.c_int, [C.c_void_p, C.c_uint32, C.c_int, C.c_void_p, C.c_uint64]),
    "nebula_mpm_batch_step": (C.c_int, [C.c_void_p, C.c_float, C.c_uint32, C.c_void_p]),
    "nebula_mpm_batch_set_graphs": (C.c_int, [C.c_void_p, C.c_int]),
    "nebula_mpm_batch_set_launch_config": (C.c_int, [C.c_void_p, C.c_void_p]),
    "nebula_mpm_batch_get_launch_config": (C.c_int, [C.c_void_p, C.c_void_p]),
    "nebula_mpm_batch_sync": (C.c_int, [C.c_void_p]),
    "nebula_mpm_batch_get_stats": (C.c_int, [C.c_void_p, C.POINTER(BatchStats)]),
    "nebula_mpm_batch_scene_info": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(SceneInfo)]),
    "nebula_mpm_adjoint_create": (C.c_int, [C.POINTER(AdjointConfig), C.POINTER(C.c_void_p)]),
    "nebula_mpm_adjoint_destroy": (C.c_int, [C.c_void_p]),
    "nebula_mpm_adjoint_forward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_float * 3, C.c_void_p, C.c_void_p]),
    "nebula_mpm_adjoint_backward": (C.c_int, [C.c_void_p, C.c_float, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "nebula_mpm_adjoint_download": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_uint64]),
    "nebula_mpm_adjoint_events": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint32)]),
    "nebula_mpm_adjoint_set_graphs": (C.c_int, [C.c_void_p, C.c_int]),
    "nebula_mpm_adjoint_launches": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64)]),
    "nebula_mpm_domain_grid_res": (None, [C.c_float * 3, C.c_float, C.c_uint32 * 3]),
    "nebula_mpm_domain_cube_res": (C.c_uint32, [C.c_uint32 * 3]),
    "nebula_mpm_domain_hash_cells": (C.c_uint32, [C.c_uint32 * 3]),
    "nebula_mpm_domain_n_groups": (C.c_uint32, [C.c_uint32]),
    "nebula_mpm_bin_workspace_size": (C.c_size_t, [C.c_uint32, C.c_uint32]),
    "nebula_hash_bin_workspace_size": (C.c_size_t, [C.c_uint32, C.c_uint32]),
    "nebula_hash_bin": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t,
                                  C.c_void_p]),
    "nebula_mpm_bin": (C.c_int, [C.POINTER(Pass), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p]),
    "nebula_mpm_bin_noalloc_max_cells": (C.c_size_t, []),
    "nebula_mpm_bin_noalloc_max_particles": (C.c_size_t, []),
    "nebula_mpm_bin_noalloc": (C.c_int, [C.POINTER(Pass), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "nebula_mpm_bin_status": (C.c_int, [C.c_void_p, C.c_size_t, C.c_uint32, C.c_uint32, C.POINTER(C.c_uint32), C.c_void_p]),
    "nebula_mpm_bin_probe_wait_expiry": (C.c_int, [C.POINTER(Pass), C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p]),
    "nebula_mpm_bin_noalloc_status": (C.c_int, [C.POINTER(C.c_uint32), C.c_void_p]),
    "nebula_mpm_bin_noalloc_probe_wait_expiry": (C.c_int, [C.POINTER(Pass), C.c_void_p, C.c_void_p]),
    "nebula_mpm_p2g": (C.c_int, [C.POINTER(Pass), C.POINTER(Particles), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                 C.c_void_p, C.c_void_p]),
    "nebula_mpm_grid_update": (C.c_int, [C.POINTER(Pass), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "nebula_mpm_g2p": (C.c_int, [C.POINTER(Pass), C.POINTER(Particles), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
}

# every exported symbol the header declares
EXPORTED = tuple(_SIGS)


def lib() -> C.CDLL:
    """Load libnebula_mpm.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError("libnebula_mpm.so is missing: run `python -m nebula_b200.build` (nvcc, sm_100a); "
                              "there is no CPU fallback")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    m = lib().nebula_mpm_last_error()
    return m.decode() if m else ""


def call(name: str, *args) -> int:
    """Call a status-returning entry point; raise NebulaError on failure."""
    rc = getattr(lib(), name)(*args)
    if rc != OK:
        raise NebulaError(rc, last_error())
    return rc
