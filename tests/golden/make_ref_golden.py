#!/usr/bin/env python3
"""Generate tests/golden/ref_shader_fixtures.npz from the reference's own shaders.

The reference's MPM compute shaders, compiled for the CPU by
oracle/build_ref.py from the reference tree (oracle/_ref/libref_mpm.so), are
run on seeded scenes that together take every branch of the substep:

  * elastic shear block under APIC, with the four analytic colliders (moving)
    and a wind beside gravity;
  * Drucker-Prager shear block under FLIP 0.7;
  * Von Mises shear block under PIC;
  * VISCOPLASTIC_MUD and FLUID shear blocks under APIC;
  * a Drucker-Prager slab sunk into the terrain SDF on 64^3 (grid SDF boundary
    and particle push-out).

For each: every 32nd particle's full state (x, v, F, B with their w lanes) as
float32, and float64 sums of every field over all particles.  The fixture
lets the oracle be checked against the reference's outputs bit for bit where
the reference tree is absent (tests/test_golden.py).

Run:  python tests/golden/make_ref_golden.py   (needs the reference tree)
"""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from nebula_b200 import scenes as S  # noqa: E402
from oracle import ref as R  # noqa: E402

OUT = Path(__file__).resolve().parent / "ref_shader_fixtures.npz"
EVERY = 32


def colliders():
    box = np.zeros(1, S.COLLIDER_DTYPE)
    box["type"], box["pos"], box["nrm"], box["vel"], box["restitution"], box["friction"] = 2, (0.42, 0.62, 0.5), (0.03, 0.05, 0.2), (0, 0.5, 0), 0.5, 0.1
    plane = np.zeros(1, S.COLLIDER_DTYPE)
    plane["type"], plane["pos"], plane["nrm"], plane["restitution"], plane["friction"] = 0, (0, 0.6, 0), (0.2, 1.0, 0.0), 0.0, 0.5
    cap = np.zeros(1, S.COLLIDER_DTYPE)
    cap["type"], cap["pos"], cap["nrm"], cap["radius"], cap["friction"] = 3, (0.58, 0.7, 0.3), (0.0, 0.0, 0.4), 0.03, 0.2
    return [S.sphere_collider((0.5, 0.78, 0.5), 0.06, vel=(0.0, -1.0, 0.0), restitution=0.2, friction=0.3), box[0], plane[0], cap[0]]


def cases():
    """(name, scene, substeps) of every case; the tests build the same scenes."""
    a = S.shear_block(S.MAT_ELASTIC)
    a.params.colliders = colliders()
    a.params.forces = [S.gravity(), S.wind((0.3, 0.0, 1.0), 2.0, affect_mask=1)]
    slab = S.slope_flow(res=64, n_side=(60, 6, 60), substeps=40, dt=1e-4, lift=-1.0)
    return [("elastic_colliders_apic", a, 30),
            ("drucker_prager_flip", S.shear_block(S.MAT_DRUCKER_PRAGER, flip_ratio=0.7), 30),
            ("von_mises_pic", S.shear_block(S.MAT_VON_MISES, flip_ratio=0.0), 30),
            ("mud_apic", S.shear_block(S.MAT_VISCOPLASTIC_MUD), 30),
            ("fluid_apic", S.shear_block(S.MAT_FLUID), 30),
            ("terrain_slab_64", slab, 40)]


def pack(st):
    return np.concatenate([np.asarray(st[f], np.float32)[::EVERY] for f in S.FIELDS], axis=1)


def sums(st):
    return np.array([np.asarray(st[f], np.float64).sum(axis=0) for f in S.FIELDS])


def main():
    if not R.available():
        sys.exit("the reference tree (or an earlier build of oracle/_ref) is needed")
    out = {}
    for name, sc, n in cases():
        r = R.RefShaders(4)
        r.set_params(sc.params)
        r.set_sdf(sc.sdf)
        r.set_state(sc.state)
        r.run(n)
        st = r.get_state()
        out[name + "_every32"] = pack(st)
        out[name + "_sums"] = sums(st)
        out[name + "_substeps"] = np.int32(n)
        print(name, sc.n, "particles,", n, "substeps")
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, OUT.stat().st_size, "bytes")


if __name__ == "__main__":
    main()
