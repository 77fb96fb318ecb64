"""The float64 adjoint oracle (oracle/mpm_adjoint.cpp) on the CPU.

It is the reference gradient for the CUDA adjoint, so it is pinned here
against central finite differences of its own float64 forward: the Hencky
stress VJP on random deformation gradients, and the rollout gradient on a
216-particle block that lands on the floor (contact through the wall band),
with eps = 1e-7 (larger steps cross the wall band's kinks) and the
jump-robust slope of oracle.fd_slope (the forward has sparse small jumps
where a grid node's mass crosses the 1e-10 activation threshold).
"""
import numpy as np

import oracle


def test_hencky_vjp_matches_fd():
    rng = np.random.default_rng(7)
    for _ in range(20):
        F = np.eye(3) + 0.3 * rng.standard_normal((3, 3))
        if np.linalg.det(F) < 0.2:
            continue
        mu, lam = 3e3, 5e3
        tb = rng.standard_normal((3, 3))
        Fb, mb, lb = oracle.hencky_ref64_vjp(F, mu, lam, tb)
        eps = 1e-6
        fd = np.zeros((3, 3))
        for i in range(3):
            for j in range(3):
                d = np.zeros((3, 3))
                d[i, j] = eps
                fd[i, j] = np.sum(tb * (oracle.hencky_ref64(F + d, mu, lam) - oracle.hencky_ref64(F - d, mu, lam))) / (2 * eps)
        assert np.allclose(Fb, fd, rtol=1e-5, atol=1e-4)
        fmu = np.sum(tb * (oracle.hencky_ref64(F, mu + 1e-3, lam) - oracle.hencky_ref64(F, mu - 1e-3, lam))) / 2e-3
        flam = np.sum(tb * (oracle.hencky_ref64(F, mu, lam + 1e-3) - oracle.hencky_ref64(F, mu, lam - 1e-3))) / 2e-3
        assert abs(mb - fmu) <= 1e-6 * max(1.0, abs(fmu))
        assert abs(lb - flam) <= 1e-6 * max(1.0, abs(flam))


def tiny(y0=0.16, vy=-2.0, seed=2):
    rng = np.random.default_rng(seed)
    res, h, n = (16, 16, 16), 1 / 16, 216
    g = np.stack(np.meshgrid(*[np.arange(6)] * 3, indexing="ij"), -1).reshape(-1, 3)
    x0 = np.array([0.4, y0, 0.4]) + g * 0.5 * h + rng.uniform(-0.1, 0.1, (n, 3)) * h
    v0 = np.array([0.3, vy, -0.2]) + rng.uniform(-0.05, 0.05, (n, 3))
    Vp = np.full(n, (0.5 * h) ** 3)
    rho = np.full(n, 1000.0)
    E = np.exp(rng.uniform(np.log(5e3), np.log(5e4), n))
    mu, lam = E / 2.6, E * 0.3 / (1.3 * 0.4)
    params = {"dt": 2e-4, "h": h, "g": (0, -9.8, 0)}
    return params, res, x0, v0, Vp, rho, mu, lam, np.array([0.5, 0.5, 0.5])


def test_rollout_gradient_matches_fd_with_floor_contact():
    a = tiny()
    params, res, x0, v0, Vp, rho, mu, lam, target = a
    nsub = 120
    r = oracle.adjoint_grad(*a, nsub, every=20)
    assert r["events"] == 0
    assert r["xT"][:, 1].min() < 2.5 * params["h"]  # the block reached the floor band
    rng = np.random.default_rng(3)
    eps = 1e-7
    for k in range(4):
        dv = rng.standard_normal(v0.shape)
        fd, _ = oracle.fd_slope(lambda t: oracle.adjoint_loss(params, res, x0, v0 + t * dv, Vp, rho, mu, lam, target, nsub)[0], eps)
        assert abs(np.sum(r["gv0"] * dv) - fd) <= 1e-4 * abs(fd)
    for k in range(2):
        dl = rng.standard_normal(mu.shape)
        fd, _ = oracle.fd_slope(
            lambda t: oracle.adjoint_loss(params, res, x0, v0, Vp, rho, mu * np.exp(t * dl), lam * np.exp(t * dl), target, nsub)[0], eps)
        ad = np.sum((r["gmu"] * mu + r["glam"] * lam) * dl)
        assert abs(ad - fd) <= 1e-3 * abs(fd)


def test_no_contact_means_no_dependence_on_E():
    """In free fall internal forces conserve momentum: dL/dE vanishes."""
    a = tiny(y0=0.5)
    r = oracle.adjoint_grad(*a, 60, every=20)
    mu, lam = a[6], a[7]
    scale = np.linalg.norm(r["gv0"])
    assert np.linalg.norm(r["gmu"] * mu) < 1e-8 * scale and np.linalg.norm(r["glam"] * lam) < 1e-8 * scale


def test_checkpoint_interval_does_not_change_gradient():
    a = tiny()
    r1 = oracle.adjoint_grad(*a, 50, every=1)
    r2 = oracle.adjoint_grad(*a, 50, every=20)
    assert np.array_equal(r1["gv0"], r2["gv0"]) and np.array_equal(r1["gmu"], r2["gmu"])
