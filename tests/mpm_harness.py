"""Per-pass harness for the known-answer tests, over two backends.

Mirrors tests/helpers/MPMHarness.{h,cpp} of the reference: a cubic grid of
``grid_res`` cells over ``[0, world]^3``, ``makePC(dt, rho0, mu, lam, gravity)``
defaults (PIC, one ELASTIC material, one gravity force along +y with the given
signed strength, MPMHarness.cpp:192-251), and per-pass runners.

* ``OracleBackend`` drives the CPU oracle (test infrastructure);
* ``GpuBackend`` drives the CUDA single-pass C ABI (``nebula_b200.passes``).
"""
from __future__ import annotations

import numpy as np

from nebula_b200.scenes import (FIELDS, FORCE_DTYPE, MAT_ELASTIC, MATERIAL_DTYPE, StepParams, morton_encode)


def harness_params(grid_res=8, world=10.0, dt=0.001, rho0=1000.0, mu=5000.0, lam=11538.0, gravity=0.0, flip_ratio=0.0) -> StepParams:
    """MPMHarness::makePC (MPMHarness.cpp:192-251)."""
    m = np.zeros(1, MATERIAL_DTYPE)
    m["mu"], m["lambda"], m["rho0"], m["model"], m["q_max"] = mu, lam, rho0, MAT_ELASTIC, 1e5
    f = np.zeros(1, FORCE_DTYPE)
    f["type"] = 0
    f["data"][0, :4] = (0.0, 1.0, 0.0, gravity)
    h = float(np.float32(world) / np.float32(grid_res))
    sp = StepParams(dt=dt, cell_size=h, domain_size=(world, world, world), flip_ratio=flip_ratio, materials=[m[0]], forces=[f[0]])
    sp.mu_lame, sp.lambda_lame, sp.rho0 = mu, lam, rho0
    sp.M_friction, sp.q_cohesion, sp.q_max = 0.577, 0.0, 1e5
    return sp


def particles(items):
    """items: list of dicts with pos, Vp, vel, F (3x3 GLSL [c][r]) and tau."""
    n = len(items)
    st = {f: np.zeros((n, 4), np.float32) for f in FIELDS}
    for i, p in enumerate(items):
        F = np.asarray(p.get("F", np.eye(3)), np.float32)
        tau = np.asarray(p.get("tau", np.zeros((3, 3))), np.float32)
        st["P"][i, :3] = p["pos"]
        st["P"][i, 3] = p.get("Vp", 1.0)
        st["v"][i, :3] = p.get("vel", (0, 0, 0))
        st["v"][i, 3] = np.uint32(p.get("mat", 0)).view(np.float32)
        st["F0"][i] = (*F[0], tau[0][0])
        st["F1"][i] = (*F[1], tau[1][1])
        st["F2"][i] = (*F[2], tau[2][2])
        st["B0"][i, 3] = tau[0][1]
        st["B1"][i, 3] = tau[0][2]
        st["B2"][i, 3] = tau[1][2]
    return st


def read_F(st, i):
    return np.stack([st["F0"][i, :3], st["F1"][i, :3], st["F2"][i, :3]])  # [c][r]


def read_stress(st, i):
    """MPMHarness::readParticleStress (MPMHarness.cpp:375-391), [c][r]."""
    txx, tyy, tzz = st["F0"][i, 3], st["F1"][i, 3], st["F2"][i, 3]
    txy, txz, tyz = st["B0"][i, 3], st["B1"][i, 3], st["B2"][i, 3]
    return np.array([[txx, txy, txz], [txy, tyy, tyz], [txz, tyz, tzz]])


def mcode(x, y, z):
    return int(morton_encode(np.array([x]), np.array([y]), np.array([z]))[0])


class OracleBackend:
    name = "oracle"

    def __init__(self, sp: StepParams, n: int, mode="ref32"):
        from oracle import Oracle
        self.o = Oracle(mode)
        self.sp = sp
        self.n = n
        self.o.set_params(sp)
        self.nc = sp.hash_cells

    def set_params(self, sp):
        self.sp = sp
        self.o.set_params(sp)

    def upload_particles(self, st):
        self.o.set_state(st)

    def upload_grid(self, mom, mass):
        full = np.zeros((2 * self.nc, 4), np.float32)
        m = np.asarray(mom, np.float32).reshape(-1, 4)
        full[: m.shape[0]] = m
        self.o.set_grid(full, mass)

    def bin(self):
        self.o.bin()

    def p2g(self):
        self.o.zero_grid()
        self.o.p2g()

    def grid_update(self):
        self.o.grid_update()
        self.o.sdf_bc()

    def g2p(self):
        self.o.g2p()

    def full_step(self):
        self.o.substep()

    def read_state(self):
        s = self.o.get_state()
        out = {f: s[f].astype(np.float32) for f in FIELDS}
        out["v"][:, 3] = s["mat"].view(np.float32)
        return out

    def read_grid(self):
        mom, mass = self.o.get_grid()
        return mom.astype(np.float32), mass.astype(np.float32)

    def read_bins(self):
        return self.o.get_bins()


class GpuBackend:
    name = "gpu"

    def __init__(self, sp: StepParams, n: int):
        from nebula_b200.passes import PassRunner
        self.r = PassRunner(sp, n)
        self.sp = sp
        self.n = n
        self.nc = sp.hash_cells

    def set_params(self, sp):
        self.sp = sp
        self.r.set_params(sp)

    def upload_particles(self, st):
        self.r.upload_particles(st)

    def upload_grid(self, mom, mass):
        self.r.upload_grid(mom, mass)

    def bin(self):
        self.r.bin()

    def p2g(self):
        self.r.p2g()

    def grid_update(self):
        self.r.grid_update()

    def g2p(self):
        self.r.g2p()

    def full_step(self):
        self.r.full_step()

    def read_state(self):
        return self.r.read_state()

    def read_grid(self):
        return self.r.read_grid()

    def read_bins(self):
        return self.r.read_bins()
