"""The reference's own MPM shaders, run on the CPU -- TEST INFRASTRUCTURE ONLY.

ctypes driver of ``oracle/_ref/libref_mpm.so`` (built by ``oracle/build_ref.py``
from the reference's shader sources).  ``RefShaders`` has the per-pass
interface of ``oracle.Oracle`` and ``hash_bin`` the interface of
``oracle.hash_bin``, so a test can run each on the same inputs and compare;
only ``tests/`` and ``bench.py --impl reference`` use them.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import FIELDS, make_params
from .build_ref import DEFAULT_REFERENCE, LIB, build

_lib = None


def available(reference: Path = DEFAULT_REFERENCE, prebuilt: bool = False) -> bool:
    """True when the library exists or can be built from the reference tree
    (with ``prebuilt``: only when it exists; the reference tree is not looked
    at)."""
    if prebuilt:
        return LIB.exists()
    try:
        return build(reference) is not None
    except Exception:
        return False


def lib():
    global _lib
    if _lib is None:
        path = LIB if LIB.exists() else build()
        if path is None:
            raise RuntimeError("reference shader library not built and the reference tree is absent")
        L = C.CDLL(str(path))
        vp = C.c_void_p
        L.ref_create.restype = vp
        L.ref_create.argtypes = []
        for name, args in [
            ("ref_destroy", [vp]),
            ("ref_set_threads", [vp, C.c_int]),
            ("ref_set_intended_scan", [vp, C.c_int]),
            ("ref_set_params", [vp, vp]),
            ("ref_set_tables", [vp, vp, C.c_uint32, vp, C.c_uint32, vp, C.c_uint32]),
            ("ref_set_sdf", [vp, vp]),
            ("ref_set_state", [vp, vp, C.c_uint32]),
            ("ref_get_state", [vp, vp]),
            ("ref_set_grid", [vp, vp, vp]),
            ("ref_get_grid", [vp, vp, vp]),
            ("ref_set_bins", [vp, vp, vp, vp]),
            ("ref_get_bins", [vp, vp, vp, vp]),
            ("ref_zero_grid", [vp]),
            ("ref_bin", [vp]),
            ("ref_p2g", [vp]),
            ("ref_grid_update", [vp]),
            ("ref_sdf_bc", [vp]),
            ("ref_g2p", [vp]),
            ("ref_substep", [vp]),
            ("ref_run", [vp, C.c_uint32]),
            ("ref_hash_bin", [vp, vp, C.c_uint32, vp, C.c_float, vp, C.c_uint32, vp, vp, vp]),
        ]:
            f = getattr(L, name)
            f.argtypes = args
            f.restype = None
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


class RefShaders:
    """One scene run through the reference's shaders on the CPU (float32, as
    the shaders compute).  ``intended_scan``: the binning's scan passes give
    the plain exclusive prefix over any number of cells, as they intend (the
    reference's own single 1024-wide global scan is wrong above 262,144
    cells); every compiled shader is unchanged either way."""

    def __init__(self, threads: int = 1, intended_scan: bool = False):
        self._L = lib()
        self._h = self._L.ref_create()
        self._L.ref_set_threads(self._h, threads)
        self._L.ref_set_intended_scan(self._h, int(intended_scan))
        self.n = 0
        self.nc = 0
        self._keep = []

    def close(self):
        if self._h:
            self._L.ref_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, sp):
        p = make_params(sp)
        self._L.ref_set_params(self._h, C.byref(p))
        self.nc = sp.hash_cells
        mats = np.ascontiguousarray(sp.materials_array())
        cols = np.ascontiguousarray(sp.colliders_array())
        frc = np.ascontiguousarray(sp.forces_array())
        self._keep = [mats, cols, frc]
        self._L.ref_set_tables(self._h, _ptr(mats), len(sp.materials), _ptr(cols), len(sp.colliders), _ptr(frc),
                               len(sp.forces))

    def set_sdf(self, sdf):
        if sdf is None:
            self._L.ref_set_sdf(self._h, None)
        else:
            s = np.ascontiguousarray(sdf, dtype=np.float32)
            assert s.size == self.nc
            self._L.ref_set_sdf(self._h, _ptr(s))

    def set_state(self, st: dict):
        arrs = [np.ascontiguousarray(st[f], dtype=np.float32).reshape(-1, 4) for f in FIELDS]
        self.n = arrs[0].shape[0]
        table = (C.c_void_p * 8)(*[a.ctypes.data for a in arrs])
        self._L.ref_set_state(self._h, C.cast(table, C.c_void_p), self.n)

    def get_state(self) -> dict:
        out = {f: np.empty((self.n, 4), np.float32) for f in FIELDS}
        table = (C.c_void_p * 8)(*[out[f].ctypes.data for f in FIELDS])
        self._L.ref_get_state(self._h, C.cast(table, C.c_void_p))
        out["mat"] = out["v"][:, 3].view(np.uint32).copy()
        return out

    def set_grid(self, mom, mass):
        m = np.ascontiguousarray(mom, dtype=np.float32).reshape(-1)
        s = np.ascontiguousarray(mass, dtype=np.float32).reshape(-1)
        assert m.size == 8 * self.nc and s.size == self.nc
        self._L.ref_set_grid(self._h, _ptr(m), _ptr(s))

    def get_grid(self):
        mom = np.empty((2 * self.nc, 4), np.float32)
        mass = np.empty(self.nc, np.float32)
        self._L.ref_get_grid(self._h, _ptr(mom), _ptr(mass))
        return mom, mass

    def set_bins(self, cnt, off, srt):
        c = np.ascontiguousarray(cnt, dtype=np.uint32)
        o = np.ascontiguousarray(off, dtype=np.uint32)
        s = np.ascontiguousarray(srt, dtype=np.uint32)
        self._L.ref_set_bins(self._h, _ptr(c), _ptr(o), _ptr(s))

    def get_bins(self):
        cnt = np.empty(self.nc, np.uint32)
        off = np.empty(self.nc, np.uint32)
        srt = np.empty(self.n, np.uint32)
        self._L.ref_get_bins(self._h, _ptr(cnt), _ptr(off), _ptr(srt))
        return cnt, off, srt

    def zero_grid(self):
        self._L.ref_zero_grid(self._h)

    def bin(self):
        self._L.ref_bin(self._h)

    def p2g(self):
        self._L.ref_p2g(self._h)

    def grid_update(self):
        self._L.ref_grid_update(self._h)

    def sdf_bc(self):
        self._L.ref_sdf_bc(self._h)

    def g2p(self):
        self._L.ref_g2p(self._h)

    def substep(self):
        self._L.ref_substep(self._h)

    def run(self, nsub: int):
        self._L.ref_run(self._h, nsub)


def hash_bin(pred_p, type_flag, world_min, cell_size: float, grid_res, hash_cells: int, sorted_init=0xFFFFFFFF):
    """The PBF engine's spatial hash run through the reference's own
    hash_count.comp / hash_sort.comp: (cellCount, cellOffset = range ends,
    sortedIdx), with the arguments and results of ``oracle.hash_bin``."""
    p = np.ascontiguousarray(pred_p, np.float32).reshape(-1, 4)
    n = p.shape[0]
    tf = None if type_flag is None else np.ascontiguousarray(type_flag, np.uint32)
    wm = np.ascontiguousarray(world_min, np.float32)
    gr = np.ascontiguousarray(grid_res, np.uint32)
    cnt = np.empty(int(hash_cells), np.uint32)
    off = np.empty(int(hash_cells), np.uint32)
    srt = np.full(n, sorted_init, np.uint32)
    lib().ref_hash_bin(_ptr(p), None if tf is None else _ptr(tf), n, _ptr(wm), C.c_float(cell_size), _ptr(gr), int(hash_cells),
                       _ptr(cnt), _ptr(off), _ptr(srt))
    return cnt, off, srt
