"""Build the reference's own MPM compute shaders as a CPU library -- TEST INFRASTRUCTURE ONLY.

The reference runs its MPMEngine substep as GLSL compute shaders through
Vulkan, which cannot run on this machine.  The shaders themselves are plain
per-invocation code (no shared memory, barriers or subgroup operations; P2G is
a per-node gather, the only atomics are the integer counters of the hash
count / sort), so this recipe compiles them with g++ against
``oracle/glsl_compat.hpp`` and links them with ``oracle/ref_dispatch.cpp``, a
dispatcher that issues the passes in the order of ``MPMEngine::step``.  The
result, ``oracle/_ref/libref_mpm.so``, is the checker of the CPU restatement
in ``oracle/mpm_oracle.cpp`` (``tests/test_ref_shaders.py``) and the CPU arm of
``bench.py --impl reference``; nothing in ``nebula_b200`` touches it.

The shader sources are read where they lie in the reference tree (default
``/root/reference``, or ``--reference DIR``); nothing of them is committed.
Every rewrite below is mechanical and changes no arithmetic:

* comments and the ``#version`` / ``#extension`` lines are dropped;
* ``#include "x"`` points at the rewritten copy of ``x``;
* the bindless ``buffers[]`` declaration and ``layout(local_size_x = ...) in;``
  are dropped (``glsl_env.hpp`` declares the buffer table), and the push-constant block becomes a struct of the same
  layout (188 bytes, asserted);
* ``out`` / ``inout`` parameters become C++ references (arrays: references
  to arrays);
* unsuffixed floating literals get an ``f`` (GLSL floating literals are
  float);
* ``.xyz`` becomes ``.xyz()`` (the only swizzle the shaders use);
* ``void main()`` becomes ``void shader_main(uvec3 gl_GlobalInvocationID)``:
  the built-in input is the entry point's parameter.

``mpm_grid_update.comp`` carries a FORCE_AUTOGEN placeholder that the
reference fills at run time (``src/core/ForceShaderCompiler.cpp:71-93,
126-139``): the velocity-force call block replaces the marker lines and every
force type's GLSL function (``src/core/Force.h``, the ``glslApplyVelocity``
raw strings) is inserted before ``void main(``.  This recipe does the same
with every force type that has a velocity function, reading the functions,
type numbers and variable lists out of ``Force.h``.

The three hash-scan shaders use workgroup shared memory and barriers; the
dispatcher restates them (``ref_dispatch.cpp``), keeping their single
1024-wide global scan.  The PBF engine's spatial hash (``hash_count.comp``,
``hash_sort.comp`` on ``common.glsl``) is built the same way, for the checker
of ``nebula_hash_bin``.
"""
from __future__ import annotations

import argparse
import os
import re
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
GEN = OUT / "gen"
LIB = OUT / "libref_mpm.so"
DEFAULT_REFERENCE = Path("/root/reference")

# The MPM passes of MPMEngine::step (src/engine/MPMEngine.cpp:418-471) that run
# as per-invocation shaders, and whether their invocations are independent
# (so a dispatch may spread them over threads).
SHADERS = {
    "mpm_zero_grid.comp": True,
    "mpm_hash_count.comp": False,
    "mpm_hash_sort.comp": False,
    "mpm_p2g.comp": True,
    "mpm_grid_update.comp": True,
    "mpm_nanovdb_bc.comp": True,
    "mpm_g2p.comp": True,
    # the PBF engine's spatial hash (Engine's hash build), on common.glsl's SimPC
    "hash_count.comp": False,
    "hash_sort.comp": False,
}
INCLUDES = ("mpm_common.glsl", "collider_common.glsl", "force_common.glsl", "force_noise.glsl", "common.glsl")
# push-constant block sizes: MPMSimPC (mpm_common.glsl) and SimPC (common.glsl)
PC_BYTES = {"mpm": 188, "hash": 200}

_FLOAT_LIT = re.compile(r"(?<![\w.])((?:\d+\.\d*|\.\d+)(?:[eE][+-]?\d+)?|\d+[eE][+-]?\d+)(?![\w.])")


def strip_comments(src: str) -> str:
    src = re.sub(r"/\*.*?\*/", " ", src, flags=re.S)
    return re.sub(r"//[^\n]*", "", src)


def rewrite(src: str) -> str:
    """The mechanical GLSL -> C++ rewrites listed in the module docstring."""
    src = strip_comments(src)
    src = re.sub(r"^[ \t]*#[ \t]*(version|extension)\b[^\n]*$", "", src, flags=re.M)
    src = re.sub(r'^([ \t]*#[ \t]*include[ \t]*)"([^"]+)"', r'\1"\2.hpp"', src, flags=re.M)
    src = re.sub(r"layout\s*\([^)]*\)\s*buffer\s+\w+\s*\{[^}]*\}\s*buffers\s*\[\s*\]\s*;", "", src)
    src = re.sub(r"layout\s*\([^)]*\)\s*in\s*;", "", src)
    src = re.sub(r"layout\s*\(\s*push_constant\s*\)\s*uniform\s+(\w+)", r"struct \1", src)
    src = re.sub(r"\b(?:inout|out)\s+(\w+)\s+(\w+)\s*\[(\d+)\]", r"\1 (&\2)[\3]", src)
    src = re.sub(r"\b(?:inout|out)\s+(\w+)\s+(\w+)", r"\1& \2", src)
    src = re.sub(r"\bvoid\s+main\s*\(\s*\)", "void shader_main(uvec3 gl_GlobalInvocationID)", src)
    src = _FLOAT_LIT.sub(r"\1f", src)
    src = re.sub(r"\.xyz\b(?!\s*\()", ".xyz()", src)
    return src


def velocity_forces(force_h: str):
    """(type number, suffix, variables, GLSL function) of every force type with
    a ``glslApplyVelocity`` body, read out of ``src/core/Force.h``."""
    enum = re.search(r"enum\s+class\s+ForceType[^{]*\{([^}]*)\}", force_h)
    numbers = {m.group(1): int(m.group(2)) for m in re.finditer(r"(\w+)\s*=\s*(\d+)u?", enum.group(1))}
    out = []
    for m in re.finditer(r"struct\s+(\w+)\s*:\s*public\s+Force\s*\{", force_h):
        body = force_h[m.end():]
        nxt = re.search(r"\nstruct\s+\w+\s*:\s*public\s+Force", body)
        body = body[: nxt.start()] if nxt else body
        vel = re.search(r"glslApplyVelocity\(\)\s*const\s*override\s*\{\s*return\s+R\"\((.*?)\)\";", body, re.S)
        if not vel:
            continue
        ftype = re.search(r"ForceType::(\w+)", body).group(1)
        suffix = re.search(r"glslFunctionSuffix\(\)\s*const\s*override\s*\{\s*return\s+\"(\w+)\"", body).group(1)
        vars_ = re.search(r"variables\(\)\s*const\s*override\s*\{(.*?)\n\s*\}", body, re.S)
        variables = [(v.group(1), v.group(2), int(v.group(3)))
                     for v in re.finditer(r"\{\s*\"(\w+)\"\s*,\s*ForceVar::(\w+)\s*,\s*(\d+)\s*\}", vars_.group(1))] if vars_ else []
        out.append((numbers[ftype], suffix, variables, vel.group(1)))
    return sorted(out)


def force_call_block(forces) -> str:
    """The velocity-force loop that replaces the FORCE_AUTOGEN marker lines
    (restates ForceShaderCompiler::buildVelocityCallBlock and argExpr,
    src/core/ForceShaderCompiler.cpp:43-52,71-93)."""
    acc = {"FLOAT": "FORCE_DATA_FLOAT", "VEC3": "FORCE_DATA_VEC3", "UINT": "FORCE_DATA_UINT"}
    lines = ["    {", "        vec3 fVel = v.xyz;", "        for (uint fi = 0u; fi < pc.forceCount; fi++) {",
             "            uint fbase = fi * 8u;", "            uint ftype = FORCE_TYPE_AT(pc.forceBufIdx, fbase);",
             "            uint fmask = FORCE_AFFECT_MASK(pc.forceBufIdx, fbase);",
             "            if (fmask != 0u && ((fmask >> forceTypeFlag) & 1u) == 0u) continue;"]
    for number, suffix, variables, _ in forces:
        args = "".join(", %s(pc.forceBufIdx, fbase, %du)" % (acc[k], off) for _, k, off in variables)
        lines += ["            if (ftype == %du) {" % number,
                  "                forceApplyVelocity_%s(fVel, forcePos, forceTypeFlag, pc.dt%s);" % (suffix, args),
                  "            }"]
    lines += ["        }", "        v.xyz = fVel;", "    }"]
    return "\n".join(lines) + "\n"


def splice_forces(src: str, forces) -> str:
    """ForceShaderCompiler::compile's two edits (src/core/ForceShaderCompiler.cpp:126-139)."""
    b = src.find("FORCE_AUTOGEN_BEGIN")
    e = src.find("FORCE_AUTOGEN_END")
    assert 0 <= b < e, "FORCE_AUTOGEN markers not found"
    line_start = src.rfind("\n", 0, b) + 1
    line_end = src.find("\n", e)
    src = src[:line_start] + force_call_block(forces) + src[line_end + 1:]
    m = src.find("void main(")
    assert m >= 0
    return src[:m] + "".join(f[3] + "\n" for f in forces) + "\n" + src[m:]


WRAPPER = """// generated by oracle/build_ref.py from the reference's %(shader)s -- test infrastructure only
#include "glsl_compat.hpp"
namespace %(ns)s {
#include "%(shader)s.hpp"
static_assert(sizeof(PC) == %(pcbytes)d, "push-constant layout");
}  // namespace %(ns)s
extern "C" void ref_run_%(ns)s(const void* pc, uint32_t count, int threads) {
  __builtin_memcpy(&%(ns)s::pc, pc, sizeof(%(ns)s::pc));
%(pragma)s  for (int64_t i = 0; i < int64_t(count); ++i) %(ns)s::shader_main(uvec3(uint(i), 0u, 0u));
}
"""


def generate(reference: Path) -> list:
    shaders = reference / "shaders"
    GEN.mkdir(parents=True, exist_ok=True)
    forces = velocity_forces((reference / "src" / "core" / "Force.h").read_text())
    for inc in INCLUDES:
        (GEN / (inc + ".hpp")).write_text(rewrite((shaders / inc).read_text()))
    wrappers = []
    for shader, independent in SHADERS.items():
        src = (shaders / shader).read_text()
        if "FORCE_AUTOGEN_BEGIN" in src:
            src = splice_forces(src, forces)
        (GEN / (shader + ".hpp")).write_text(rewrite(src))
        ns = shader.split(".")[0]
        w = GEN / ("ref_%s.cpp" % ns)
        pragma = "#pragma omp parallel for schedule(dynamic, 4096) num_threads(threads > 0 ? threads : 1)\n" if independent else ""
        w.write_text(WRAPPER % {"shader": shader, "ns": ns, "pragma": pragma, "pcbytes": PC_BYTES[ns.split("_")[0]]})
        wrappers.append(w)
    return wrappers


def build(reference: Path = DEFAULT_REFERENCE, force: bool = False):
    """Compile ``oracle/_ref/libref_mpm.so``; returns its path, or None when
    neither the reference tree nor an earlier build is present."""
    have_ref = (reference / "shaders" / "mpm_g2p.comp").exists()
    if not have_ref:
        return LIB if LIB.exists() else None
    deps = [HERE / "glsl_compat.hpp", HERE / "glsl_env.hpp", HERE / "ref_dispatch.cpp", Path(__file__)]
    if LIB.exists() and not force and all(LIB.stat().st_mtime >= d.stat().st_mtime for d in deps):
        return LIB
    wrappers = generate(reference)
    tmp = LIB.with_suffix(".so.tmp%d" % os.getpid())
    cmd = ["g++", "-O2", "-std=c++17", "-fopenmp", "-ffp-contract=off", "-fno-strict-aliasing", "-fPIC", "-shared",
           "-w", "-I", str(HERE), "-I", str(GEN), "-o", str(tmp), str(HERE / "ref_dispatch.cpp")] + [str(w) for w in wrappers]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--reference", type=Path, default=DEFAULT_REFERENCE)
    a = ap.parse_args()
    p = build(a.reference, force=True)
    print(p if p else "reference tree not found: nothing built")
    sys.exit(0 if p else 1)
