"""The header-only C++ facade (include/nebula_mpm.hpp) with the reference's
MPMEngine method names: it compiles warning-free against the library and
reports failures as exceptions (CPU); on a GPU it steps like the Python
binding of the same C ABI."""
import json
import subprocess
from pathlib import Path

import numpy as np
import pytest

from nebula_b200 import build

ROOT = Path(__file__).resolve().parent.parent


def compile_demo(tmp_path) -> Path:
    build.build()
    exe = tmp_path / "facade_demo"
    lib = ROOT / "nebula_b200"
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", str(ROOT / "include"), str(ROOT / "tests" / "cpp" / "facade_demo.cpp"),
                    "-L", str(lib), "-lnebula_mpm", "-Wl,-rpath," + str(lib), "-o", str(exe)], check=True)
    return exe


def run_demo(exe) -> dict:
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    return json.loads(out.stdout.strip().splitlines()[-1])


def test_facade_compiles_and_reports_errors(tmp_path):
    r = run_demo(compile_demo(tmp_path))
    assert "ok" in r
    if not r["ok"]:
        assert r["error"].startswith("nebula_mpm: ")


@pytest.mark.gpu
def test_facade_steps_like_the_python_binding(tmp_path):
    r = run_demo(compile_demo(tmp_path))
    assert r["ok"] and r["live"] == 32 ** 3
    from nebula_b200 import scenes as S
    from nebula_b200.engine import MPMConfig, MPMEngine
    eng = MPMEngine(MPMConfig())
    eng.addForce(S.gravity())
    eng.flip_ratio = -1.0
    eng.numSubsteps = 10
    for _ in range(2):
        eng.step(1e-3)
    mean = eng.download("P")[:, :3].astype(np.float64).mean(axis=0)
    assert np.allclose(r["mean"], mean, rtol=0, atol=1e-6)
