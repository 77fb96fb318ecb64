"""Known-answer tests of the reference, restated (tests/test_mpm.cpp, tests/test_domain.cpp).

Each pass-level KAT runs on two backends: the CPU oracle (pins the oracle to
the reference's own expectations; no GPU) and the CUDA single-pass ABI
(marked ``gpu``).  Tolerances are the reference's.
"""
import math

import numpy as np
import pytest

from mpm_harness import (GpuBackend, OracleBackend, harness_params, mcode, particles, read_F, read_stress)
from nebula_b200 import scenes as S

BACKENDS = [pytest.param("oracle", id="oracle"), pytest.param("gpu", id="gpu", marks=pytest.mark.gpu)]


@pytest.fixture(params=BACKENDS)
def backend(request):
    def make(sp, n):
        return OracleBackend(sp, n) if request.param == "oracle" else GpuBackend(sp, n)
    return make


# ----------------------------------------------------------------------------- CPU math (test_mpm.cpp:59-168)
def test_partition_of_unity():
    """1-1 (test_mpm.cpp:59-92): 27 weights sum to 1 within 1e-5."""
    import oracle
    h = 1.25
    offs = [0.1, 0.3, 0.6, 0.9, 1.1]
    for ox in offs:
        for oy in offs:
            for oz in offs:
                xp = np.float32([(2 + ox) * h, (2 + oy) * h, (2 + oz) * h])
                base = np.floor(xp / np.float32(h)).astype(int) - 1
                s = 0.0
                for iz in range(3):
                    for iy in range(3):
                        for ix in range(3):
                            n = base + np.array([ix, iy, iz])
                            d = (xp - (n + 0.5) * np.float32(h)) / np.float32(h)
                            s += oracle.bspline2(d[0]) * oracle.bspline2(d[1]) * oracle.bspline2(d[2])
                assert abs(s - 1.0) < 1e-5


def test_gradient_sum_zero():
    """1-2 (test_mpm.cpp:98-132): sum of weight gradients is 0 within 1e-5."""
    import oracle
    h = 1.25
    offs = [0.2, 0.5, 0.8, 1.2]
    for ox in offs:
        for oy in offs:
            for oz in offs:
                xp = np.float32([(3 + ox) * h, (3 + oy) * h, (3 + oz) * h])
                base = np.floor(xp / np.float32(h)).astype(int) - 1
                g = np.zeros(3)
                for iz in range(3):
                    for iy in range(3):
                        for ix in range(3):
                            n = base + np.array([ix, iy, iz])
                            d = (xp - (n + 0.5) * np.float32(h)) / np.float32(h)
                            w = [oracle.bspline2(v) for v in d]
                            dg = [oracle.bspline2g(v) for v in d]
                            g += [dg[0] * w[1] * w[2], w[0] * dg[1] * w[2], w[0] * w[1] * dg[2]]
                assert np.all(np.abs(g) < 1e-5)


def test_hencky_identity_zero():
    """5-1 (test_mpm.cpp:137-144): F = I gives zero stress."""
    import oracle
    t = oracle.hencky(np.eye(3), 5000.0, 11538.0)
    assert np.all(np.abs(t) < 1e-4)


@pytest.mark.parametrize("fp64", [False, True])
def test_hencky_uniform_compression(fp64):
    """5-2 (test_mpm.cpp:149-168): F = 0.9 I -> (3 lam + 2 mu) ln 0.9 on the diagonal."""
    import oracle
    mu, lam = 5000.0, 11538.0
    t = oracle.hencky(0.9 * np.eye(3), mu, lam, fp64=fp64)
    exp = (3 * lam + 2 * mu) * math.log(0.9)
    assert t[0, 0] < -1 and t[1, 1] < -1 and t[2, 2] < -1
    assert abs(t[0, 0] - t[1, 1]) < 1 and abs(t[1, 1] - t[2, 2]) < 1
    assert abs(t[0, 1]) < 1e-4 and abs(t[0, 2]) < 1e-4 and abs(t[1, 2]) < 1e-4
    assert abs(t[0, 0] - exp) < abs(exp) * 0.01


def _fixed_corotated_np(F, mu, lam):
    """tau = 2 mu (F - R) F^T + lam (J - 1) J I in float64, R the rotation of
    F's polar decomposition (det R = +1 also for an inverted F), written from
    numpy's SVD independently of the oracle's Jacobi svd3."""
    U, s, Vt = np.linalg.svd(F)
    if np.linalg.det(U) < 0:
        U[:, 2] *= -1
        s[2] *= -1
    if np.linalg.det(Vt) < 0:
        Vt[2, :] *= -1
        s[2] *= -1
    R = U @ Vt
    J = np.linalg.det(F)
    return 2 * mu * (F - R) @ F.T + lam * (J - 1) * J * np.eye(3)


@pytest.mark.parametrize("fp64", [False, True])
def test_fixed_corotated_stress_matches_polar_formula(fp64):
    """Model 6: the oracle's stress (svd3 + diagonal form) against the polar
    formula, for random stretches, rotations and an inverted F; zero at F = I
    and at any pure rotation."""
    import oracle
    mu, lam = 3846.15, 5769.23
    rng = np.random.default_rng(11)
    for k in range(40):
        F = np.eye(3) + 0.3 * rng.standard_normal((3, 3))
        if k == 39:
            F = np.diag([1.05, 0.95, -0.9]) @ F  # inverted
        if abs(np.linalg.det(F)) < 0.2:
            continue
        want = _fixed_corotated_np(F, mu, lam)
        got = oracle.fixed_corotated(F.T, mu, lam, fp64=fp64).T  # GLSL layout is column-major
        assert np.allclose(got, want, rtol=0, atol=(1e-6 if fp64 else 2e-2) * max(1.0, np.abs(want).max())), k
    assert np.all(np.abs(oracle.fixed_corotated(np.eye(3), mu, lam)) < 1e-3)
    c, s = np.cos(0.7), np.sin(0.7)
    Rz = np.array([[c, -s, 0], [s, c, 0], [0, 0, 1]])
    assert np.all(np.abs(oracle.fixed_corotated(Rz.T, mu, lam, fp64=True)) < 1e-3)
    # small axis-aligned strains: both models linearise to lam tr(e) I + 2 mu e
    F = np.diag([1.001, 0.999, 1.0005])
    fc, he = oracle.fixed_corotated(F, mu, lam, fp64=True), oracle.hencky(F, mu, lam, fp64=True)
    assert np.allclose(fc, he, rtol=3e-3, atol=1e-3)


# ----------------------------------------------------------------------------- domain (test_domain.cpp:8-50)
def test_domain_grid_res():
    assert S.grid_res((10.0, 10.0, 10.0), 10.0 / 64.0) == (64, 64, 64)
    assert S.grid_res((10.0, 10.0, 10.0), 3.0) == (4, 4, 4)
    assert S.grid_res((40.0, 10.0, 10.0), 5.0) == (8, 2, 2)
    assert S.grid_res((0.01,) * 3, 5.0) == (1, 1, 1)
    assert S.grid_res((0.0,) * 3, 5.0) == (1, 1, 1)


def test_domain_cube_res_and_hash_cells():
    assert S.morton_cube_res((64, 64, 64)) == 64
    assert S.morton_cube_res((5, 5, 5)) == 8
    assert S.morton_cube_res((40, 10, 10)) == 64
    assert S.morton_cube_res((1, 1, 1)) == 1
    assert S.hash_cells((64, 64, 64)) == 64 ** 3
    hc = S.hash_cells((40, 10, 10))
    assert hc == 64 ** 3 and hc > 40 * 10 * 10
    assert S.n_groups(256) == 1 and S.n_groups(257) == 2 and S.n_groups(0) == 0


# ----------------------------------------------------------------------------- pass KATs (test_mpm.cpp:236-396)
def test_p2g_mass_momentum(backend):
    """2-1 (test_mpm.cpp:236-271): one particle, mass 1.5, momentum (3, -1.5, 0)."""
    sp = harness_params(8, 10.0, dt=0.001, rho0=1.0)
    b = backend(sp, 1)
    b.upload_particles(particles([dict(pos=(5.0, 5.0, 5.0), Vp=1.5, vel=(2.0, -1.0, 0.0))]))
    b.bin()
    b.p2g()
    mom, mass = b.read_grid()
    nc = sp.hash_cells
    assert abs(mass.sum() - 1.5) < 1e-3
    m = mom[:nc, :3].astype(np.float64).sum(0)
    assert abs(m[0] - 3.0) < 1e-2 and abs(m[1] + 1.5) < 1e-2 and abs(m[2]) < 1e-2


def test_grid_update_gravity(backend):
    """3-1 (test_mpm.cpp:276-303): v.y = -9.8 * 0.01 at an interior node."""
    sp = harness_params(8, 10.0, dt=0.01, rho0=1000.0, gravity=-9.8)
    b = backend(sp, 1)
    nc = sp.hash_cells
    t = mcode(4, 4, 4)
    mom = np.zeros((nc, 4), np.float32)
    mass = np.zeros(nc, np.float32)
    mass[t] = 1.0
    b.upload_grid(mom, mass)
    b.grid_update()
    g, _ = b.read_grid()
    v = g[t, :3]
    assert abs(v[0]) < 1e-4 and abs(v[1] + 0.098) < 1e-4 and abs(v[2]) < 1e-4


def test_grid_update_wall(backend):
    """3-2 (test_mpm.cpp:309-339): inward normal velocity removed at ix = 1."""
    sp = harness_params(8, 10.0, dt=0.01, gravity=0.0)
    b = backend(sp, 1)
    nc = sp.hash_cells
    t = mcode(1, 4, 4)
    mom = np.zeros((nc, 4), np.float32)
    mass = np.zeros(nc, np.float32)
    mass[t] = 1.0
    mom[t] = (-5.0, 2.0, 0.0, 0.0)
    b.upload_grid(mom, mass)
    b.grid_update()
    g, _ = b.read_grid()
    v = g[t, :3]
    assert abs(v[0]) < 1e-4 and abs(v[1] - 2.0) < 1e-4 and abs(v[2]) < 1e-4


def test_g2p_uniform_field(backend):
    """4-1 (test_mpm.cpp:345-396): a uniform grid velocity is reproduced."""
    sp = harness_params(8, 10.0, dt=0.001)
    h = sp.cell_size
    b = backend(sp, 1)
    b.upload_particles(particles([dict(pos=(5.1, 5.1, 5.1), Vp=1.0)]))
    nc = sp.hash_cells
    base = int(np.floor(np.float32(5.1) / np.float32(h))) - 1
    mom = np.zeros((nc, 4), np.float32)
    mass = np.zeros(nc, np.float32)
    U = (1.5, 3.0, 0.0)
    for iz in range(3):
        for iy in range(3):
            for ix in range(3):
                m = mcode(base + ix, base + iy, base + iz)
                mass[m] = 1.0
                mom[m, :3] = U
    b.upload_grid(mom, mass)
    b.g2p()
    v = b.read_state()["v"][0, :3]
    assert np.all(np.abs(v - np.array(U)) < 1e-3)


# ----------------------------------------------------------------------------- integration (test_mpm.cpp:402-743)
def test_full_step_50_no_nan_in_bounds(backend):
    """6-1 (test_mpm.cpp:402-457)."""
    sp = harness_params(16, 10.0, dt=1.0 / (60.0 * 4.0), rho0=1000.0, mu=1e4, lam=2.3e4, gravity=-9.8)
    s = 0.3
    items = []
    for iz in range(2):
        for iy in range(2):
            for ix in range(2):
                items.append(dict(pos=(5 + (ix - 0.5) * s, 7 + (iy - 0.5) * s, 5 + (iz - 0.5) * s), Vp=s ** 3))
    b = backend(sp, 8)
    b.upload_particles(particles(items))
    for _ in range(50):
        b.full_step()
    st = b.read_state()
    lo, hi = sp.cell_size * 1.5, 10.0 - sp.cell_size * 1.5
    assert np.all(np.isfinite(st["P"][:, :3])) and np.all(np.isfinite(st["v"][:, :3]))
    assert np.all(st["P"][:, :3] >= lo) and np.all(st["P"][:, :3] <= hi)


def test_single_particle_constant_velocity(backend):
    """6-2 (test_mpm.cpp:463-507): PIC keeps one particle's velocity across cells."""
    sp = harness_params(8, 10.0, dt=0.01, rho0=1.0)
    b = backend(sp, 1)
    b.upload_particles(particles([dict(pos=(4.2, 5.0, 5.0), Vp=1.0, vel=(1.0, 0.0, 0.0))]))
    for _ in range(20):
        b.full_step()
        v = b.read_state()["v"][0]
        assert abs(v[0] - 1.0) < 1e-3 and abs(v[1]) < 1e-3
    x = b.read_state()["P"][0, 0]
    assert abs(x - (4.2 + 20 * 0.01)) < 0.05


def test_full_pipeline_gravity_one_step(backend):
    """7-1 (test_mpm.cpp:519-557): v = g dt and x advanced by dt v."""
    sp = harness_params(8, 10.0, dt=0.01, rho0=1000.0, gravity=-9.8)
    h = sp.cell_size
    b = backend(sp, 1)
    b.upload_particles(particles([dict(pos=(5.0, 5.0, 5.0), Vp=h ** 3)]))
    b.full_step()
    st = b.read_state()
    v, x = st["v"][0, :3], st["P"][0, :3]
    assert abs(v[0]) < 1e-4 and abs(v[1] + 0.098) < 1e-4 and abs(v[2]) < 1e-4
    assert abs(x[0] - 5) < 1e-4 and abs(x[1] - (5 + 0.01 * -0.098)) < 1e-4 and abs(x[2] - 5) < 1e-4


def test_g2p_velocity_gradient_updates_F(backend):
    """7-2 (test_mpm.cpp:567-630): v_x = A (x_i - x_p) gives F = diag(1 + A dt, 1, 1)."""
    sp = harness_params(8, 10.0, dt=0.01)
    h = sp.cell_size
    b = backend(sp, 1)
    b.upload_particles(particles([dict(pos=(5.0, 5.0, 5.0), Vp=1.0)]))
    A = 10.0
    base = int(np.floor(np.float32(5.0) / np.float32(h))) - 1
    nc = sp.hash_cells
    mom = np.zeros((nc, 4), np.float32)
    mass = np.zeros(nc, np.float32)
    for iz in range(3):
        for iy in range(3):
            for ix in range(3):
                nx = base + ix
                m = mcode(nx, base + iy, base + iz)
                xi = (nx + 0.5) * h
                mom[m, 0] = A * (xi - 5.0)
                mass[m] = 1.0
    b.upload_grid(mom, mass)
    b.g2p()
    st = b.read_state()
    F = read_F(st, 0)
    assert abs(F[0, 0] - (1 + A * 0.01)) < 2e-3
    assert abs(F[1, 1] - 1) < 1e-4 and abs(F[2, 2] - 1) < 1e-4
    for (i, j) in [(0, 1), (1, 0), (0, 2), (2, 0)]:
        assert abs(F[i, j]) < 1e-4
    t = read_stress(st, 0)
    assert t[0, 0] > 0 and t[1, 1] > 0 and t[0, 0] > t[1, 1] + 100.0 and abs(t[0, 1]) < 1.0


def test_momentum_conservation(backend):
    """7-3 (test_mpm.cpp:638-688): PIC, no forces, tau = 0 conserves momentum."""
    sp = harness_params(8, 10.0, dt=0.01, rho0=1.0)
    items = [dict(pos=(4, 5, 5), vel=(2, 0, 0)), dict(pos=(6, 5, 5), vel=(-2, 0, 0)),
             dict(pos=(5, 4, 5), vel=(0, 2, 0)), dict(pos=(5, 6, 5), vel=(0, -2, 0))]
    for it in items:
        it["Vp"] = 0.3
    b = backend(sp, 4)
    b.upload_particles(particles(items))
    b.full_step()
    v = b.read_state()["v"][:, :3].astype(np.float64)
    tot = (0.3 * v).sum(0)
    assert np.all(np.abs(tot) < 1e-3)


def test_wall_clamp(backend):
    """7-4 (test_mpm.cpp:696-743): a particle fired at the x wall stays inside."""
    sp = harness_params(8, 10.0, dt=0.01, rho0=1000.0, mu=1e4, lam=2.3e4)
    h = sp.cell_size
    lo = 1.5 * h
    b = backend(sp, 1)
    b.upload_particles(particles([dict(pos=(2.5, 5.0, 5.0), Vp=h ** 3, vel=(-5.0, 0.0, 0.0))]))
    for _ in range(30):
        b.full_step()
        assert b.read_state()["P"][0, 0] >= lo - 1e-4
    v = b.read_state()["v"][0, :3]
    assert v[0] >= -0.5 and np.all(np.isfinite(v))
