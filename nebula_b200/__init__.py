"""nebula_b200 -- B200-native MLS-MPM substep behind nebula's MPMEngine surface.

The compute path is hand-written sm_100a CUDA in ``csrc/`` built into
``libnebula_mpm.so`` (C ABI: ``include/nebula_mpm.h``).  Python is a thin
ctypes binding used by tests and the benchmark:

* ``engine.MPMEngine`` -- the reference's ``MPMEngine`` surface;
* ``passes``           -- single reference dispatches on device buffers;
* ``scenes``           -- seeded synthetic workloads and parameter records;
* ``build``            -- nvcc build of the shared library.
"""
from .scenes import (COLLIDER_DTYPE, FIELDS, FORCE_DTYPE, MATERIAL_DTYPE, StepParams, Scene, gravity, lame, material,
                     sphere_collider)

__all__ = ["COLLIDER_DTYPE", "FIELDS", "FORCE_DTYPE", "MATERIAL_DTYPE", "StepParams", "Scene", "gravity", "lame", "material",
           "sphere_collider"]
