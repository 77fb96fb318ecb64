"""CPU oracle for the MPMEngine substep -- TEST INFRASTRUCTURE ONLY.

This package is the parity checker for the CUDA path and the timed CPU
baseline.  Only ``tests/``, ``bench.py`` (its ``cpu_baseline`` leg and the
``--impl reference`` arm) and ``__graft_entry__.smoke()`` may import it; the
product package ``nebula_b200`` never does.

``mpm_oracle.cpp`` restates the reference's shaders (see its header for the
file:line map) in C++ templated on precision; this module builds it with g++
and drives it through ctypes.  Modes:

* ``"ref32"`` -- float everywhere, the shaders' own precision and algorithm;
* ``"mixed"`` -- float state, float64 SVD/stress inside the plastic return
  maps (the CUDA path's precision policy);
* ``"fp64"``  -- float64 everywhere (error statements, finite differences).

``ref32`` is pinned bit for bit to the reference's own shaders compiled for
the CPU (``oracle/build_ref.py``, driven by ``oracle/ref.py``;
``tests/test_ref_shaders.py`` and the golden vectors of
``tests/golden/ref_shader_fixtures.npz``).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SRC = HERE / "mpm_oracle.cpp"
SRCS = (HERE / "mpm_oracle.cpp", HERE / "mpm_adjoint.cpp", HERE / "mpm_emit_oracle.cpp", HERE / "mpm_mesh_sdf_oracle.cpp",
        HERE / "hash_bin_oracle.cpp")
LIB = HERE / "libmpm_oracle.so"

MODES = {"ref32": 0, "mixed": 1, "fp64": 2}
FIELDS = ("P", "v", "F0", "F1", "F2", "B0", "B1", "B2")


class orc_params(C.Structure):
    _fields_ = [
        ("dt", C.c_float),
        ("cellSize", C.c_float),
        ("gridRes", C.c_uint32 * 3),
        ("hashCells", C.c_uint32),
        ("worldMin", C.c_float * 3),
        ("worldMax", C.c_float * 3),
        ("flip_ratio", C.c_float),
        ("materialCount", C.c_uint32),
        ("mu_lame", C.c_float),
        ("lambda_lame", C.c_float),
        ("rho0", C.c_float),
        ("M_friction", C.c_float),
        ("q_cohesion", C.c_float),
        ("q_max", C.c_float),
        ("plasticModel", C.c_uint32),
        ("colliderCount", C.c_uint32),
        ("forceCount", C.c_uint32),
    ]


def build(force: bool = False) -> Path:
    """Compile the oracle into ``oracle/libmpm_oracle.so`` (g++, OpenMP)."""
    if LIB.exists() and not force and all(LIB.stat().st_mtime >= s.stat().st_mtime for s in SRCS):
        return LIB
    tmp = LIB.with_suffix(".so.tmp%d" % os.getpid())
    cmd = ["g++", "-O2", "-std=c++17", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared",
           "-o", str(tmp)] + [str(s) for s in SRCS]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        vp = C.c_void_p
        L.orc_create.restype = vp
        L.orc_create.argtypes = [C.c_int]
        for name, args in [
            ("orc_destroy", [vp]),
            ("orc_set_params", [vp, C.POINTER(orc_params)]),
            ("orc_set_tables", [vp, vp, C.c_uint32, vp, C.c_uint32, vp, C.c_uint32]),
            ("orc_set_sdf", [vp, vp]),
            ("orc_set_state", [vp] + [vp] * 8 + [C.c_uint32]),
            ("orc_get_state", [vp] + [vp] * 8),
            ("orc_get_mat_ids", [vp, vp]),
            ("orc_set_grid", [vp, vp, vp]),
            ("orc_get_grid", [vp, vp, vp]),
            ("orc_set_bins", [vp, vp, vp, vp]),
            ("orc_get_bins", [vp, vp, vp, vp]),
            ("orc_zero_grid", [vp]),
            ("orc_bin", [vp]),
            ("orc_p2g", [vp]),
            ("orc_grid_update", [vp]),
            ("orc_sdf_bc", [vp]),
            ("orc_g2p", [vp]),
            ("orc_substep", [vp]),
            ("orc_run", [vp, C.c_uint32]),
            ("orc_set_num_threads", [C.c_int]),
            ("orc_morton_decode", [C.c_uint32, vp]),
            ("orc_hencky", [vp, C.c_float, C.c_float, vp, C.c_int]),
            ("orc_fixed_corotated", [vp, C.c_float, C.c_float, vp, C.c_int]),
            ("orc_svd3", [vp, vp, vp, vp]),
            ("orc_project", [vp, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, vp]),
        ]:
            f = getattr(L, name)
            f.argtypes = args
            f.restype = None
        L.adj_grad.restype = C.c_int
        L.adj_grad.argtypes = [vp, vp, C.c_size_t] + [vp] * 7 + [C.c_int, C.c_int] + [vp] * 6
        L.adj_loss.restype = C.c_int
        L.adj_loss.argtypes = [vp, vp, C.c_size_t] + [vp] * 7 + [C.c_int, vp, vp]
        L.adj_hencky.restype = None
        L.adj_hencky.argtypes = [vp, C.c_double, C.c_double, vp]
        L.adj_hencky_vjp.restype = None
        L.adj_hencky_vjp.argtypes = [vp, C.c_double, C.c_double, vp, vp, vp, vp]
        L.orc_num_threads.restype = C.c_int
        L.orc_bspline2.restype = C.c_float
        L.orc_bspline2.argtypes = [C.c_float]
        L.orc_bspline2g.restype = C.c_float
        L.orc_bspline2g.argtypes = [C.c_float]
        L.orc_morton_encode.restype = C.c_uint32
        L.orc_morton_encode.argtypes = [C.c_uint32] * 3
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def make_params(sp) -> orc_params:
    """Build ``orc_params`` from a ``nebula_b200.scenes.StepParams``-like object."""
    p = orc_params()
    p.dt = sp.dt
    p.cellSize = sp.cell_size
    p.gridRes[:] = list(sp.grid_res)
    p.hashCells = sp.hash_cells
    p.worldMin[:] = list(sp.world_min)
    p.worldMax[:] = list(sp.world_max)
    p.flip_ratio = sp.flip_ratio
    p.materialCount = len(sp.materials)
    p.mu_lame = sp.mu_lame
    p.lambda_lame = sp.lambda_lame
    p.rho0 = sp.rho0
    p.M_friction = sp.M_friction
    p.q_cohesion = sp.q_cohesion
    p.q_max = sp.q_max
    p.plasticModel = sp.plastic_model
    p.colliderCount = len(sp.colliders)
    p.forceCount = len(sp.forces)
    return p


class Oracle:
    """One simulated scene on the CPU oracle."""

    def __init__(self, mode: str = "ref32"):
        self._L = lib()
        self._h = self._L.orc_create(MODES[mode])
        self.mode = mode
        self.n = 0
        self.nc = 0
        self._keep = []

    def close(self):
        if self._h:
            self._L.orc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---------------------------------------------------------------- setup
    def set_params(self, sp):
        p = make_params(sp)
        self._L.orc_set_params(self._h, C.byref(p))
        self.nc = sp.hash_cells
        mats = np.ascontiguousarray(sp.materials_array())
        cols = np.ascontiguousarray(sp.colliders_array())
        frc = np.ascontiguousarray(sp.forces_array())
        self._keep = [mats, cols, frc]
        self._L.orc_set_tables(self._h, _ptr(mats), len(sp.materials), _ptr(cols), len(sp.colliders),
                               _ptr(frc), len(sp.forces))

    def set_sdf(self, sdf):
        if sdf is None:
            self._L.orc_set_sdf(self._h, None)
        else:
            s = np.ascontiguousarray(sdf, dtype=np.float32)
            assert s.size == self.nc
            self._L.orc_set_sdf(self._h, _ptr(s))

    def set_state(self, st: dict):
        arrs = [np.ascontiguousarray(st[f], dtype=np.float32).reshape(-1, 4) for f in FIELDS]
        n = arrs[0].shape[0]
        self.n = n
        self._L.orc_set_state(self._h, *[_ptr(a) for a in arrs], n)

    def get_state(self) -> dict:
        out = {f: np.empty((self.n, 4), np.float64) for f in FIELDS}
        self._L.orc_get_state(self._h, *[_ptr(out[f]) for f in FIELDS])
        ids = np.empty(self.n, np.uint32)
        self._L.orc_get_mat_ids(self._h, _ptr(ids))
        out["mat"] = ids
        return out

    def set_grid(self, mom, mass):
        m = np.ascontiguousarray(mom, dtype=np.float32).reshape(-1)
        s = np.ascontiguousarray(mass, dtype=np.float32).reshape(-1)
        assert m.size == 8 * self.nc and s.size == self.nc
        self._L.orc_set_grid(self._h, _ptr(m), _ptr(s))

    def get_grid(self):
        mom = np.empty((2 * self.nc, 4), np.float64)
        mass = np.empty(self.nc, np.float64)
        self._L.orc_get_grid(self._h, _ptr(mom), _ptr(mass))
        return mom, mass

    def set_bins(self, cnt, off, srt):
        c = np.ascontiguousarray(cnt, dtype=np.uint32)
        o = np.ascontiguousarray(off, dtype=np.uint32)
        s = np.ascontiguousarray(srt, dtype=np.uint32)
        self._L.orc_set_bins(self._h, _ptr(c), _ptr(o), _ptr(s))

    def get_bins(self):
        cnt = np.empty(self.nc, np.uint32)
        off = np.empty(self.nc, np.uint32)
        srt = np.empty(self.n, np.uint32)
        self._L.orc_get_bins(self._h, _ptr(cnt), _ptr(off), _ptr(srt))
        return cnt, off, srt

    # ---------------------------------------------------------------- passes
    def zero_grid(self):
        self._L.orc_zero_grid(self._h)

    def bin(self):
        self._L.orc_bin(self._h)

    def p2g(self):
        self._L.orc_p2g(self._h)

    def grid_update(self):
        self._L.orc_grid_update(self._h)

    def sdf_bc(self):
        self._L.orc_sdf_bc(self._h)

    def g2p(self):
        self._L.orc_g2p(self._h)

    def substep(self):
        self._L.orc_substep(self._h)

    def run(self, nsub: int):
        self._L.orc_run(self._h, int(nsub))


def set_num_threads(n: int):
    lib().orc_set_num_threads(int(n))


def num_threads() -> int:
    return int(lib().orc_num_threads())


def bspline2(d: float) -> float:
    return float(lib().orc_bspline2(d))


def bspline2g(d: float) -> float:
    return float(lib().orc_bspline2g(d))


def morton_encode(x: int, y: int, z: int) -> int:
    return int(lib().orc_morton_encode(x, y, z))


def morton_decode(c: int):
    out = np.zeros(3, np.uint32)
    lib().orc_morton_decode(c, _ptr(out))
    return tuple(int(v) for v in out)


def hencky(F_glsl: np.ndarray, mu: float, lam: float, fp64: bool = False) -> np.ndarray:
    """Hencky Kirchhoff stress of a 3x3 F given in GLSL layout (F[c][r])."""
    f = np.ascontiguousarray(F_glsl, dtype=np.float32).reshape(9)
    t = np.empty(9, np.float32)
    lib().orc_hencky(_ptr(f), mu, lam, _ptr(t), int(fp64))
    return t.reshape(3, 3)


def fixed_corotated(F_glsl: np.ndarray, mu: float, lam: float, fp64: bool = False) -> np.ndarray:
    """Fixed-corotated Kirchhoff stress (model 6) of a 3x3 F in GLSL layout (F[c][r])."""
    f = np.ascontiguousarray(F_glsl, dtype=np.float32).reshape(9)
    t = np.empty(9, np.float32)
    lib().orc_fixed_corotated(_ptr(f), mu, lam, _ptr(t), int(fp64))
    return t.reshape(3, 3)


def svd3(F_glsl: np.ndarray):
    f = np.ascontiguousarray(F_glsl, dtype=np.float64).reshape(9)
    U = np.empty(9)
    V = np.empty(9)
    s = np.empty(3)
    lib().orc_svd3(_ptr(f), _ptr(U), _ptr(s), _ptr(V))
    return U.reshape(3, 3), s, V.reshape(3, 3)


def project(F_glsl: np.ndarray, model: int, mu, lam, M=0.0, qc=0.0, qmax=0.0) -> np.ndarray:
    f = np.ascontiguousarray(F_glsl, dtype=np.float64).reshape(9)
    out = np.empty(9)
    lib().orc_project(_ptr(f), model, mu, lam, M, qc, qmax, _ptr(out))
    return out.reshape(3, 3)


# ----------------------------------------------------------------------------- adjoint (float64)
EVENT_NAMES = {1: "grid speed cap", 2: "J reset", 4: "world clamp", 8: "particle left the grid interior"}


def _adj_args(params, res, x0, v0, Vp, rho, mu, lam, target):
    prm = np.array([params["dt"], params["h"], *params["g"]], np.float64)
    r = np.array(res, np.int32)
    arrs = [np.ascontiguousarray(a, np.float64) for a in (x0, v0, Vp, rho, mu, lam, target)]
    return prm, r, arrs


def adjoint_grad(params, res, x0, v0, Vp, rho, mu, lam, target, nsub, every=20):
    """Reverse-mode gradient of |COM(x_T) - target|^2 w.r.t. v0 and per-particle
    (mu, lambda), float64, with checkpoints every `every` substeps."""
    prm, r, arrs = _adj_args(params, res, x0, v0, Vp, rho, mu, lam, target)
    n = arrs[2].size
    loss = np.zeros(1)
    gv = np.zeros(3 * n)
    gmu = np.zeros(n)
    glam = np.zeros(n)
    xT = np.zeros(3 * n)
    ev = np.zeros(1, np.uint32)
    lib().adj_grad(_ptr(prm), _ptr(r), n, *[_ptr(a) for a in arrs], int(nsub), int(every), _ptr(loss), _ptr(gv), _ptr(gmu),
                   _ptr(glam), _ptr(xT), _ptr(ev))
    return {"loss": float(loss[0]), "gv0": gv.reshape(n, 3), "gmu": gmu, "glam": glam, "xT": xT.reshape(n, 3), "events": int(ev[0])}


def adjoint_loss(params, res, x0, v0, Vp, rho, mu, lam, target, nsub):
    prm, r, arrs = _adj_args(params, res, x0, v0, Vp, rho, mu, lam, target)
    n = arrs[2].size
    loss = np.zeros(1)
    ev = np.zeros(1, np.uint32)
    lib().adj_loss(_ptr(prm), _ptr(r), n, *[_ptr(a) for a in arrs], int(nsub), _ptr(loss), _ptr(ev))
    return float(loss[0]), int(ev[0])


def hencky_ref64(F, mu, lam):
    f = np.ascontiguousarray(F, np.float64).reshape(9)
    t = np.zeros(9)
    lib().adj_hencky(_ptr(f), mu, lam, _ptr(t))
    return t.reshape(3, 3)


def hencky_ref64_vjp(F, mu, lam, tbar):
    f = np.ascontiguousarray(F, np.float64).reshape(9)
    tb = np.ascontiguousarray(tbar, np.float64).reshape(9)
    fb = np.zeros(9)
    mb = np.zeros(1)
    lb = np.zeros(1)
    lib().adj_hencky_vjp(_ptr(f), mu, lam, _ptr(tb), _ptr(fb), _ptr(mb), _ptr(lb))
    return fb.reshape(3, 3), float(mb[0]), float(lb[0])


def fd_slope(loss_at, eps):
    """Derivative at t = 0 of t -> loss_at(t) from five evaluations, robust to
    an isolated jump: of the one-sided slopes on [-2e, -e], [-e, 0], [0, e],
    [e, 2e], the one farthest from their median is dropped and the median of
    the other three is returned.  The reference forward has sparse small jumps
    (a grid node whose mass crosses the 1e-10 activation threshold enters
    G2P with its stress-driven velocity), so a plain central difference that
    straddles one is meaningless; one jump spoils at most one of the four
    slopes.  Returns (median, slopes)."""
    L = {k: loss_at(k * eps) for k in (-2, -1, 0, 1, 2)}
    s = np.array([(L[-1] - L[-2]) / eps, (L[0] - L[-1]) / eps, (L[1] - L[0]) / eps, (L[2] - L[1]) / eps])
    keep = np.delete(s, np.argmax(np.abs(s - np.median(s))))
    return float(np.median(keep)), s


def emit(record, Vp: float, seed: int, event: int, n: int):
    """n emitted particles of one emission (mpm_emit_oracle.cpp): (pos4, vel4)."""
    rec = np.ascontiguousarray(np.asarray(record).reshape(-1)[:1])
    pos = np.zeros((n, 4), np.float32)
    vel = np.zeros((n, 4), np.float32)
    lib().orc_emit(rec.ctypes.data_as(C.c_void_p), C.c_float(Vp), C.c_uint64(seed), C.c_uint64(event), C.c_uint32(n),
                   pos.ctypes.data_as(C.c_void_p), vel.ctypes.data_as(C.c_void_p))
    return pos, vel


def mesh_sdf(tris, res, total_cells: int, cell_size: float, complete: bool = True):
    """buildMeshSDF restated on the CPU (mpm_mesh_sdf_oracle.cpp): Morton-ordered
    float32 SDF; complete=False reproduces the reference's closest-point steps
    (edge-BC region left out)."""
    t = np.ascontiguousarray(tris, np.float32).reshape(-1, 12)
    r = np.ascontiguousarray(res, np.uint32)
    out = np.empty(int(total_cells), np.float32)
    lib().orc_mesh_sdf(t.ctypes.data_as(C.c_void_p), C.c_uint32(t.shape[0]), r.ctypes.data_as(C.c_void_p), C.c_uint32(int(total_cells)),
                       C.c_float(cell_size), out.ctypes.data_as(C.c_void_p), C.c_int(int(bool(complete))))
    return out


def hash_bin(pred_p, type_flag, world_min, cell_size: float, grid_res, hash_cells: int, sorted_init=0xFFFFFFFF):
    """The PBF spatial hash restated on the CPU (hash_bin_oracle.cpp):
    (cellCount, cellOffset = range ends, sortedIdx).  pred_p: (n, 4) float32;
    type_flag: (n,) uint32 or None.  Slots of sortedIdx past the included
    particles keep `sorted_init`."""
    p = np.ascontiguousarray(pred_p, np.float32).reshape(-1, 4)
    n = p.shape[0]
    tf = None if type_flag is None else np.ascontiguousarray(type_flag, np.uint32)
    wm = np.ascontiguousarray(world_min, np.float32)
    gr = np.ascontiguousarray(grid_res, np.uint32)
    cnt = np.empty(int(hash_cells), np.uint32)
    off = np.empty(int(hash_cells), np.uint32)
    srt = np.full(n, sorted_init, np.uint32)
    lib().orc_hash_bin(p.ctypes.data_as(C.c_void_p), None if tf is None else tf.ctypes.data_as(C.c_void_p), C.c_uint32(n),
                       wm.ctypes.data_as(C.c_void_p), C.c_float(cell_size), gr.ctypes.data_as(C.c_void_p), C.c_uint32(int(hash_cells)),
                       cnt.ctypes.data_as(C.c_void_p), off.ctypes.data_as(C.c_void_p), srt.ctypes.data_as(C.c_void_p))
    return cnt, off, srt
