#!/usr/bin/env python3
"""Generate tests/golden/oracle_fixtures.npz from the CPU oracle.

The reference's path runs only as GLSL through Vulkan (no graphics API exists
here), and its test suite (tests/test_mpm.cpp, tests/test_domain.cpp) holds
analytic known-answer tests, not stored arrays; those KATs pin the oracle in
tests/test_kat_mpm.py.  This script freezes the oracle's outputs on seeded
scenes so that both the oracle (CPU tests) and the CUDA path (GPU tests) are
checked against the same committed vectors:

  * elastic block (8,000 particles, 64^3): the full binning (non-zero cells,
    their counts and range ends, sorted particle order);
  * elastic shear block: every 16th particle's state after 20 and 100 ref32
    substeps, plus float64 sums of every field over all particles;
  * jelly + sand scene (80,000 particles, 128^3): every 80th particle's x and v
    after 20 substeps in the mixed precision policy.

Run:  python tests/golden/make_golden.py
"""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from nebula_b200 import scenes as S  # noqa: E402

OUT = Path(__file__).resolve().parent / "oracle_fixtures.npz"


def run(sc, n, mode):
    o = oracle.Oracle(mode)
    o.set_params(sc.params)
    o.set_sdf(sc.sdf)
    o.set_state(sc.state)
    if n:
        o.run(n)
    return o


def pack_state(st, every):
    return np.concatenate([st[f][::every] for f in S.FIELDS], axis=1).astype(np.float32)


def sums(st):
    return np.array([st[f].astype(np.float64).sum(axis=0) for f in S.FIELDS])


def main():
    oracle.build()
    d = {}
    sc = S.elastic_block()
    o = run(sc, 0, "ref32")
    o.bin()
    cnt, off, srt = o.get_bins()
    nz = np.nonzero(cnt)[0].astype(np.uint32)
    d["bins_cells"], d["bins_count"], d["bins_end"], d["bins_sorted"] = nz, cnt[nz], off[nz], srt

    sh = S.shear_block()
    for n in (20, 100):
        st = run(sh, n, "ref32").get_state()
        d["shear_ref32_%d" % n] = pack_state(st, 16)
        d["shear_ref32_%d_sums" % n] = sums(st)

    mm = S.multimaterial()
    st = run(mm, 20, "mixed").get_state()
    d["multimaterial_mixed_20_x"] = st["P"][::80, :3].astype(np.float32)
    d["multimaterial_mixed_20_v"] = st["v"][::80, :3].astype(np.float32)
    np.savez_compressed(OUT, **d)
    print("wrote", OUT, OUT.stat().st_size, "bytes")


if __name__ == "__main__":
    main()
