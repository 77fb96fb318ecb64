"""The CUDA adjoint of the MPM rollout (nebula_mpm_adjoint_*) on the GPU.

The reference has no adjoint.  The gradient is checked against the float64
CPU adjoint (oracle/mpm_adjoint.cpp) and against float64 finite differences
of the oracle's loss on 16 seeded directions, on a 2,000-particle block in
free fall (every term at float32 precision) and pressing on the floor (where
dL/dE is not zero and the map is contact-conditioned).  The full
50,000-particle rollout is checked against a committed fixture of the
oracle's gradient projections (tests/golden/make_adjoint_golden.py).
"""
from pathlib import Path

import numpy as np
import pytest
import torch

from nebula_b200 import scenes as S
from nebula_b200.adjoint import Rollout, rollout_loss
from nebula_b200.engine import engine_for_scene

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "adjoint_diff_block_50k.npz"
SMALL = dict(n=2000, res=32, substeps=60, side=13, y0_cells=2.5, vy=-2.0)


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def inputs(sc):
    x0 = torch.from_numpy(np.ascontiguousarray(sc.state["P"])).cuda()
    v0 = torch.from_numpy(np.ascontiguousarray(sc.state["v"])).cuda()
    E = torch.from_numpy(np.ascontiguousarray(sc.extra["E"], np.float32)).cuda()
    return x0, v0, E


def oracle_args(sc, v=None, E=None):
    st = sc.state
    E = (sc.extra["E"] if E is None else E).astype(np.float64)
    nu = sc.extra["nu"]
    mu = E / (2 * (1 + nu))
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    g = sum(np.asarray(f["data"][:3], np.float64) * float(f["data"][3]) for f in sc.params.forces)
    params = {"dt": sc.params.dt, "h": sc.params.cell_size, "g": tuple(g)}
    v = st["v"][:, :3] if v is None else v
    return (params, sc.params.grid_res, st["P"][:, :3].astype(np.float64), np.asarray(v, np.float64), st["P"][:, 3].astype(np.float64),
            np.full(sc.n, sc.extra["rho0"]), mu, lam, sc.extra["target"].astype(np.float64))


def gpu_grad(sc, graphs=True):
    roll = Rollout.for_scene(sc)
    roll.set_graphs(graphs)
    x0, v0, E = inputs(sc)
    loss = roll.forward(x0, v0, E, sc.extra["target"])
    gv, gE, _ = roll.backward(1.0)
    torch.cuda.synchronize()
    return float(loss), gv[:, :3].cpu().numpy().astype(np.float64), gE.cpu().numpy().astype(np.float64), roll


def test_forward_matches_engine_uniform_E():
    """With one E for every particle the rollout's forward is the engine's substep."""
    sc = S.diff_block(**SMALL)
    sc.extra["E"] = np.full(sc.n, 1e4, np.float32)
    _, _, _, roll = gpu_grad(sc)
    eng = engine_for_scene(sc)
    eng.run_substeps(sc.params.dt, sc.substeps)
    want = eng.download("P")[:, :3]
    got = roll.final_state("P")[:, :3]
    assert rel(got, want) < 1e-5


FREE = dict(SMALL, y0_cells=12.0)  # the same block in free fall: no contact during the rollout


def test_free_fall_gradient_matches_float64_adjoint():
    """Without contact every term of the reverse pass (G2P, grid, P2G, the
    float64 Hencky VJP) is checked at float32 precision against the float64
    adjoint.  dL/dE vanishes here (momentum conservation)."""
    sc = S.diff_block(**FREE)
    import oracle
    ref = oracle.adjoint_grad(*oracle_args(sc), sc.substeps, every=20)
    L, gv, gE, roll = gpu_grad(sc)
    assert ref["events"] == 0 and roll.events() == 0
    assert abs(L - ref["loss"]) / ref["loss"] < 1e-5
    assert rel(gv, ref["gv0"]) < 1e-5


def test_contact_gradient_matches_float64_adjoint():
    """The block presses on the floor.  The reference map is ill-conditioned
    there: a grid node whose mass is near the 1e-10 activation threshold
    carries a stress-driven velocity p/m and its adjoint carries 1/m, and
    float32 and float64 rollouts activate different such nodes.  The float64
    oracle itself moves its v0 gradient by ~1e-4 for a 1e-7 relative change of
    x0 (against 1e-8 in free fall), so v0 is held to 2e-2 and E to 1e-2."""
    sc = S.diff_block(**SMALL)
    import oracle
    ref = oracle.adjoint_grad(*oracle_args(sc), sc.substeps, every=20)
    assert ref["events"] == 0
    L, gv, gE, roll = gpu_grad(sc)
    assert roll.events() == 0
    nu = sc.extra["nu"]
    gE_ref = ref["gmu"] / (2 * (1 + nu)) + ref["glam"] * nu / ((1 + nu) * (1 - 2 * nu))
    assert abs(L - ref["loss"]) / ref["loss"] < 1e-5
    assert rel(gv, ref["gv0"]) < 2e-2
    assert rel(gE, gE_ref) < 1e-2
    # the block presses on the floor, so E changes the loss
    assert abs(np.sum(gE_ref * sc.extra["E"])) > 1e-4 * ref["loss"]


def test_gradient_vs_float64_fd_16_directions():
    """16 seeded directions: 8 in v0 on the free-falling block, 8 in log E on
    the block pressing on the floor; the GPU directional derivative against
    float64 finite differences of the oracle's loss (oracle.fd_slope, eps =
    1e-7: robust to the forward's sparse jumps)."""
    import oracle
    rng = np.random.default_rng(20)
    eps = 1e-7
    errs = {"v": [], "E": []}
    for name, kw in (("v", FREE), ("E", SMALL)):
        sc = S.diff_block(**kw)
        L, gv, gE, _ = gpu_grad(sc)
        E0 = sc.extra["E"].astype(np.float64)
        v0 = sc.state["v"][:, :3].astype(np.float64)
        for k in range(8):
            dv = rng.standard_normal(v0.shape) if name == "v" else np.zeros_like(v0)
            dl = rng.standard_normal(sc.n) if name == "E" else np.zeros(sc.n)
            ad = float(np.sum(gv * dv) + np.sum(gE * E0 * dl))
            fd, _ = oracle.fd_slope(lambda t: oracle.adjoint_loss(*oracle_args(sc, v=v0 + t * dv, E=E0 * np.exp(t * dl)), sc.substeps)[0], eps)
            errs[name].append(abs(ad - fd) / max(abs(fd), 1e-300))
    # the GPU v0 gradient equals the float64 adjoint to ~3e-7 here; the finite
    # differences themselves scatter by up to ~5e-4 around it
    assert max(errs["v"]) < 2e-3, errs
    assert max(errs["E"]) < 1e-2, errs


def test_autograd_function():
    sc = S.diff_block(**SMALL)
    roll = Rollout.for_scene(sc)
    x0, v0, E = inputs(sc)
    v0.requires_grad_(True)
    E.requires_grad_(True)
    loss = rollout_loss(roll, x0, v0, E, sc.extra["target"])
    (3.0 * loss).backward()
    gv, gE, _ = roll.backward(1.0)
    torch.cuda.synchronize()
    # each backward recomputes the segments; float atomics reorder the sums
    assert torch.allclose(v0.grad, 3.0 * gv, rtol=1e-3, atol=1e-3 * float(gv.abs().max()))
    assert torch.allclose(E.grad, 3.0 * gE, rtol=1e-3, atol=1e-3 * float(gE.abs().max()))


def test_graph_replay_equals_eager():
    """Same kernels replayed from graphs and launched eagerly: the same loss,
    and both gradients as close to the float64 adjoint as the contact scene
    allows (test_contact_gradient_matches_float64_adjoint).  The reductions
    into the grid are float atomics whose order changes from run to run, and
    the v0 gradient of this floor-contact scene amplifies that: graph and eager
    runs differ by 1e-4 to 5e-4 relative (measured), so they are compared
    with the reference rather than bit for bit with each other."""
    sc = S.diff_block(**SMALL)
    import oracle
    ref = oracle.adjoint_grad(*oracle_args(sc), sc.substeps, every=20)
    nu = sc.extra["nu"]
    gE_ref = ref["gmu"] / (2 * (1 + nu)) + ref["glam"] * nu / ((1 + nu) * (1 - 2 * nu))
    L1, gv1, gE1, _ = gpu_grad(sc, graphs=True)
    L2, gv2, gE2, _ = gpu_grad(sc, graphs=False)
    assert abs(L1 - L2) <= 1e-6 * abs(L2)
    for gv, gE in ((gv1, gE1), (gv2, gE2)):
        assert rel(gv, ref["gv0"]) < 2e-2 and rel(gE, gE_ref) < 1e-2
    assert rel(gv1, gv2) < 2e-3 and rel(gE1, gE2) < 2e-3


@pytest.mark.skipif(not GOLDEN.exists(), reason="fixture not generated")
def test_full_rollout_against_float64_fixture():
    """50,000 particles, 64^3, 200 substeps, checkpoints every 20: loss and the
    16 gradient projections (8 in v0, 8 in log E) against the float64 oracle's
    reverse pass and its central finite differences.

    The rollout's grid sums are float atomics whose order changes from run to
    run, and on this floor-contact scene that moves the projections by 1-2%
    between GPU runs (measured over five runs: 1.0e-2 to 1.8e-2 apart; each
    run 1.3e-2 to 2.8e-2 from the oracle, once 5.4e-2; the mean of five runs
    1.4e-2).  The bars therefore hold the mean of three runs at 4e-2, room for
    one outlying run, and each run at 8e-2."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_adjoint_golden", GOLDEN.parent / "make_adjoint_golden.py")
    gen = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gen)
    sc = S.diff_block()
    fx = np.load(GOLDEN)
    E0 = sc.extra["E"].astype(np.float64)
    dirs = [gen.directions(sc.n, k) for k in range(16)]
    runs = []
    for r in range(3):
        L, gv, gE, roll = gpu_grad(sc, graphs=(r != 1))
        assert abs(L - float(fx["loss"])) / float(fx["loss"]) < 1e-4
        proj = np.array([np.sum(gv * dv) + np.sum(gE * E0 * dl) for dv, dl in dirs])
        # log E directions: smooth at this scale, against the oracle's adjoint and its finite differences
        assert rel(proj[8:], fx["proj_adjoint"][8:]) < 8e-2 and rel(proj[8:], fx["proj_fd"][8:]) < 8e-2
        runs.append(proj)
    proj = np.mean(runs, axis=0)
    assert rel(proj[8:], fx["proj_adjoint"][8:]) < 4e-2 and rel(proj[8:], fx["proj_fd"][8:]) < 4e-2
    # v0 directions: contact-conditioned (see test_contact_gradient_matches_float64_adjoint) and the
    # loss is rough at finite-difference scale in v0 here, so only the oracle's adjoint is the reference
    assert rel(proj[:8], fx["proj_adjoint"][:8]) < 5e-2
