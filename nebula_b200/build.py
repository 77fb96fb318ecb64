"""Build the sm_100a shared library ``nebula_b200/libnebula_mpm.so`` in-tree.

All CUDA sources under ``csrc/`` are compiled by nvcc for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``) and linked into one shared
library that exports the C ABI of ``include/nebula_mpm.h``.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libnebula_mpm.so"
INCLUDE = ROOT / "include"

NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC,-O2",
    "--expt-relaxed-constexpr",
    "-Xptxas", "-O3",
]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or Path(c).exists()):
            return c
    return "nvcc"


def sources():
    return sorted(CSRC.glob("*.cu"))


def _stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = list(CSRC.glob("*")) + list(INCLUDE.glob("*.h"))
    return any(p.stat().st_mtime > t for p in deps)


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> Path:
    """Compile every .cu under csrc/ into libnebula_mpm.so (skipped when fresh)."""
    if not force and not _stale():
        return LIB
    objdir = PKG / "_build"
    objdir.mkdir(exist_ok=True)
    objs = []
    procs = []
    for src in sources():
        obj = objdir / (src.stem + ".o")
        cmd = [nvcc(), *NVCC_FLAGS, "-I", str(INCLUDE), "-c", str(src), "-o", str(obj)]
        if ptxas_info:
            cmd[1:1] = ["-Xptxas", "-v"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        procs.append((subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True), src))
        objs.append(obj)
    failed = []
    for p, src in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            failed.append((src, out))
        elif ptxas_info or verbose:
            print(out, file=sys.stderr)
    if failed:
        msg = "\n".join(f"--- {s.name}\n{o}" for s, o in failed)
        raise RuntimeError("nvcc failed:\n" + msg)
    tmp = LIB.with_name(LIB.name + ".tmp%d" % os.getpid())
    link = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-Xcompiler", "-fPIC", *map(str, objs), "-o", str(tmp)]
    if verbose:
        print(" ".join(link), file=sys.stderr)
    subprocess.run(link, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
