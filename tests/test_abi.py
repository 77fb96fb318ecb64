"""The C ABI library: builds, loads without a GPU, exports every symbol the
headers declare, and its host-only helpers match the reference's domain KATs
(tests/test_domain.cpp:8-50)."""
import ctypes as C
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


@pytest.fixture(scope="module")
def lib():
    from nebula_b200 import _capi, build
    build.build()
    return _capi.lib()


def declared_symbols():
    syms = set()
    for h in (ROOT / "include").glob("*.h"):
        txt = h.read_text()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        syms.update(re.findall(r"\b(nebula_(?:mpm|hash)_[a-z0-9_]+)\s*\(", txt))
    return sorted(syms)


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "nebula_mpm_step" in syms and "nebula_mpm_create" in syms and "nebula_mpm_g2p" in syms
    assert "nebula_hash_bin" in syms and "nebula_mpm_mesh_sdf_posed" in syms


def test_every_declared_symbol_is_exported(lib):
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_python_binding_covers_every_symbol():
    from nebula_b200 import _capi
    assert sorted(_capi.EXPORTED) == declared_symbols()


def test_domain_helpers_through_abi(lib):
    def gr(size, h):
        out = (C.c_uint32 * 3)()
        lib.nebula_mpm_domain_grid_res((C.c_float * 3)(*size), h, out)
        return tuple(out)

    assert gr((10, 10, 10), 10 / 64) == (64, 64, 64)
    assert gr((10, 10, 10), 3.0) == (4, 4, 4)
    assert gr((40, 10, 10), 5.0) == (8, 2, 2)
    assert gr((0.01,) * 3, 5.0) == (1, 1, 1)
    assert gr((0.0,) * 3, 5.0) == (1, 1, 1)
    u3 = lambda *v: (C.c_uint32 * 3)(*v)
    assert lib.nebula_mpm_domain_cube_res(u3(64, 64, 64)) == 64
    assert lib.nebula_mpm_domain_cube_res(u3(5, 5, 5)) == 8
    assert lib.nebula_mpm_domain_cube_res(u3(40, 10, 10)) == 64
    assert lib.nebula_mpm_domain_cube_res(u3(1, 1, 1)) == 1
    assert lib.nebula_mpm_domain_hash_cells(u3(40, 10, 10)) == 64 ** 3
    assert lib.nebula_mpm_domain_n_groups(256) == 1
    assert lib.nebula_mpm_domain_n_groups(257) == 2
    assert lib.nebula_mpm_domain_n_groups(0) == 0


def test_bin_workspace_size_monotone(lib):
    a = lib.nebula_mpm_bin_workspace_size(64 ** 3, 8000)
    b = lib.nebula_mpm_bin_workspace_size(128 ** 3, 80000)
    assert 0 < a < b


def test_errors_are_status_codes_not_crashes(lib):
    """Null handles and bad arguments return an error code and a message."""
    from nebula_b200 import _capi
    assert lib.nebula_mpm_step(None, C.c_float(0.01), None) == _capi.ERR_INVALID
    assert "null" in _capi.last_error()
    assert lib.nebula_mpm_create(None, None) == _capi.ERR_INVALID
    p = _capi.Pass()
    p.cellSize = 0.0
    assert lib.nebula_mpm_grid_update(C.byref(p), None, None, None, None, None, None) == _capi.ERR_INVALID


def test_create_without_device_reports_error(lib):
    """On a host without a CUDA device, create fails with a status code."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present; this case is for GPU-less hosts")
    from nebula_b200 import _capi
    from nebula_b200.engine import MPMConfig
    h = C.c_void_p()
    rc = lib.nebula_mpm_create(C.byref(MPMConfig(nx=2, ny=2, nz=2).to_c()), C.byref(h))
    assert rc in (_capi.ERR_CUDA, _capi.ERR_OOM)
    assert _capi.last_error()


def test_header_is_plain_c():
    """The boundary header compiles as C99 on its own (no C++ types cross the ABI)."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    r = subprocess.run([cc, "-x", "c", "-std=c99", "-Wall", "-Wextra", "-Werror", "-fsyntax-only", str(ROOT / "include" / "nebula_mpm.h")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
