"""Parity of the CUDA path with the CPU oracle on seeded inputs (GPU).

Bars (from the reference's own tests and the parity contract):
  * binning: cellCount, cellOffset (range end) and sorted (ascending index
    inside each cell) bit-exact;
  * P2G grid momentum / mass after one substep: relative L2 <= 1e-5 against
    the ref-fp32 oracle;
  * particle x and F after 100 substeps: relative L2 <= 1e-4 against the
    ref-fp32 oracle, with the error against the fp64 oracle printed.
"""
import numpy as np
import pytest

from mpm_harness import GpuBackend, OracleBackend
from nebula_b200 import scenes as S
from nebula_b200.engine import engine_for_scene

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def oracle_for(scene, mode="ref32"):
    from oracle import Oracle
    o = Oracle(mode)
    o.set_params(scene.params)
    o.set_sdf(scene.sdf)
    o.set_state(scene.state)
    return o


def state_F(st):
    return np.concatenate([st["F0"][:, :3], st["F1"][:, :3], st["F2"][:, :3]], axis=1)


# ----------------------------------------------------------------------------- binning
@pytest.mark.parametrize("make", [S.elastic_block, S.multimaterial], ids=["elastic_8k_64", "multimaterial_80k_128"])
def test_bins_bit_exact_engine(make):
    sc = make()
    eng = engine_for_scene(sc)
    cnt, off, srt = eng.export_bins()
    o = oracle_for(sc)
    o.bin()
    ocnt, ooff, osrt = o.get_bins()
    assert np.array_equal(cnt, ocnt)
    assert np.array_equal(off, ooff)
    assert np.array_equal(srt, osrt)


def test_bins_bit_exact_1m_256():
    """1M particles on 256^3 (16.7M cells): beyond the reference's 262,144-cell scan limit."""
    sc = S.slope_flow(with_sdf=False)
    eng = engine_for_scene(sc)
    cnt, off, srt = eng.export_bins()
    o = oracle_for(sc)
    o.bin()
    ocnt, ooff, osrt = o.get_bins()
    assert np.array_equal(cnt, ocnt) and np.array_equal(off, ooff) and np.array_equal(srt, osrt)


def test_bins_pass_api_with_outliers():
    """Particles outside the grid are clamped to boundary cells (cellIdFromPos)."""
    sc = S.elastic_block()
    st = {k: v.copy() for k, v in sc.state.items()}
    st["P"][:10, 0] = -0.3
    st["P"][10:20, 1] = 1.7
    sc.state = st
    g = GpuBackend(sc.params, sc.n)
    g.upload_particles(st)
    g.bin()
    o = OracleBackend(sc.params, sc.n)
    o.upload_particles(st)
    o.bin()
    for a, b in zip(g.read_bins(), o.read_bins()):
        assert np.array_equal(a, b)


# ----------------------------------------------------------------------------- P2G
def advanced(scene, k, mode="ref32"):
    """The scene after k oracle substeps (non-trivial F, stress and B)."""
    o = oracle_for(scene, mode)
    o.run(k)
    s = o.get_state()
    st = {f: s[f].astype(np.float32) for f in S.FIELDS}
    st["v"][:, 3] = s["mat"].view(np.float32)
    return st


@pytest.mark.parametrize("make,k", [(S.elastic_block, 0), (S.elastic_block, 30), (S.multimaterial, 20)],
                         ids=["elastic_fresh", "elastic_30", "multimaterial_20"])
def test_p2g_grid_one_substep(make, k):
    sc = make()
    if k:
        sc.state = advanced(sc, k)
    eng = engine_for_scene(sc)
    mom, mass = eng.export_grid(sc.params.dt)
    o = oracle_for(sc)
    o.zero_grid()
    o.bin()
    o.p2g()
    omom, omass = o.get_grid()
    nc = sc.params.hash_cells
    e_mom = rel_l2(mom[:, :3], omom[:nc, :3])
    e_mass = rel_l2(mass, omass)
    print("P2G rel L2: momentum %.3e mass %.3e" % (e_mom, e_mass))
    assert e_mom <= 1e-5 and e_mass <= 1e-5


# ----------------------------------------------------------------------------- grid update
def test_grid_update_colliders_sdf():
    """Random grid through walls, gravity, all four analytic colliders and a dense SDF."""
    sp = S.elastic_block().params
    rng = np.random.default_rng(7)
    sp.colliders = [S.sphere_collider((0.5, 0.3, 0.5), 0.15, vel=(0.1, 0.0, -0.2), restitution=0.2, friction=0.3)]
    box = np.zeros(1, S.COLLIDER_DTYPE)
    box["type"], box["pos"], box["nrm"], box["vel"], box["restitution"], box["friction"] = 2, (0.2, 0.6, 0.3), (0.1, 0.05, 0.1), (0, 0.3, 0), 0.5, 0.1
    plane = np.zeros(1, S.COLLIDER_DTYPE)
    plane["type"], plane["pos"], plane["nrm"], plane["restitution"], plane["friction"] = 0, (0, 0.15, 0), (0.1, 1.0, 0.0), 0.0, 0.5
    cap = np.zeros(1, S.COLLIDER_DTYPE)
    cap["type"], cap["pos"], cap["nrm"], cap["radius"], cap["friction"] = 3, (0.7, 0.4, 0.2), (0.0, 0.3, 0.4), 0.06, 0.2
    sp.colliders += [box[0], plane[0], cap[0]]
    nc = sp.hash_cells
    mass = np.where(rng.random(nc) < 0.3, rng.random(nc).astype(np.float32) * 1e-3, 0).astype(np.float32)
    mass[rng.random(nc) < 0.01] = 5e-11  # below the 1e-10 threshold
    mom = np.zeros((nc, 4), np.float32)
    mom[:, :3] = (rng.standard_normal((nc, 3)) * 2e-3).astype(np.float32)
    mom[rng.random(nc) < 0.01, :3] *= 1e4  # above the 15 m/s cap
    c = (np.arange(64) + 0.5) / 64
    X, Y, Z = np.meshgrid(c, c, c, indexing="ij")
    sdf = np.full(nc, 1e6, np.float32)
    codes = S.morton_encode(*np.meshgrid(np.arange(64), np.arange(64), np.arange(64), indexing="ij"))
    sdf[codes.ravel()] = (np.sqrt((X - 0.6) ** 2 + (Y - 0.2) ** 2 + (Z - 0.5) ** 2) - 0.2).ravel().astype(np.float32)
    g = GpuBackend(sp, 1)
    g.r.set_sdf(sdf)
    g.upload_grid(mom, mass)
    g.grid_update()
    o = OracleBackend(sp, 1)
    o.o.set_sdf(sdf)
    o.upload_grid(mom, mass)
    o.grid_update()
    gm, _ = g.read_grid()
    om, _ = o.read_grid()
    assert rel_l2(gm[:nc, :3], om[:nc, :3]) < 2e-6
    assert rel_l2(gm[nc:, :3], om[nc:, :3]) < 2e-6
    assert np.max(np.abs(gm[:nc, :3] - om[:nc, :3])) < 1e-4


# ----------------------------------------------------------------------------- G2P
@pytest.mark.parametrize("flip", [-1.0, 0.0, 0.7], ids=["apic", "pic", "flip"])
def test_g2p_pass(flip):
    sc = S.elastic_block(flip_ratio=flip)
    sc.state = advanced(sc, 20)
    o = OracleBackend(sc.params, sc.n)
    o.upload_particles(sc.state)
    o.o.zero_grid()
    o.bin()
    o.p2g()
    o.grid_update()
    mom, mass = o.read_grid()
    g = GpuBackend(sc.params, sc.n)
    g.upload_particles(sc.state)
    g.upload_grid(mom, mass)
    g.g2p()
    o.g2p()
    gs, os_ = g.read_state(), o.read_state()
    for f in S.FIELDS:
        e = rel_l2(gs[f], os_[f])
        assert e < 1e-5, (f, e)


def test_g2p_pass_plastic_mixed():
    """Drucker-Prager + Von Mises particles against the oracle in the CUDA path's
    precision policy (float state, float64 return-map SVD)."""
    sc = S.multimaterial()
    st = advanced(sc, 30, mode="mixed")
    sc.state = st
    o = OracleBackend(sc.params, sc.n, mode="mixed")
    o.upload_particles(st)
    o.o.zero_grid()
    o.bin()
    o.p2g()
    o.grid_update()
    mom, mass = o.read_grid()
    g = GpuBackend(sc.params, sc.n)
    g.upload_particles(st)
    g.upload_grid(mom, mass)
    g.g2p()
    o.g2p()
    gs, os_ = g.read_state(), o.read_state()
    assert rel_l2(gs["P"][:, :3], os_["P"][:, :3]) < 1e-6
    assert rel_l2(state_F(gs), state_F(os_)) < 1e-5
    assert rel_l2(gs["v"][:, :3], os_["v"][:, :3]) < 1e-4


# ----------------------------------------------------------------------------- trajectories
def test_trajectory_elastic_100_substeps():
    sc = S.elastic_block()
    eng = engine_for_scene(sc)
    eng.run_substeps(sc.params.dt, 100)
    gs = eng.state()
    ref = oracle_for(sc, "ref32")
    ref.run(100)
    rs = ref.get_state()
    f64 = oracle_for(sc, "fp64")
    f64.run(100)
    ds = f64.get_state()
    ex, eF = rel_l2(gs["P"][:, :3], rs["P"][:, :3]), rel_l2(state_F(gs), state_F(rs))
    ex64, eF64 = rel_l2(gs["P"][:, :3], ds["P"][:, :3]), rel_l2(state_F(gs), state_F(ds))
    print("elastic 100 substeps: x %.3e F %.3e vs ref32; x %.3e F %.3e vs fp64" % (ex, eF, ex64, eF64))
    assert ex <= 1e-4 and eF <= 1e-4


def test_trajectory_multimaterial_mixed():
    """Jelly + Drucker-Prager sand, 100 substeps, against the oracle in the same
    precision policy, with the ref-fp32 error printed."""
    sc = S.multimaterial()
    eng = engine_for_scene(sc)
    eng.run_substeps(sc.params.dt, 100)
    gs = eng.state()
    mix = oracle_for(sc, "mixed")
    mix.run(100)
    ms = mix.get_state()
    ref = oracle_for(sc, "ref32")
    ref.run(100)
    rs = ref.get_state()
    ex, eF = rel_l2(gs["P"][:, :3], ms["P"][:, :3]), rel_l2(state_F(gs), state_F(ms))
    rx, rF = rel_l2(gs["P"][:, :3], rs["P"][:, :3]), rel_l2(state_F(gs), state_F(rs))
    print("multimaterial 100 substeps: x %.3e F %.3e vs mixed; x %.3e F %.3e vs ref32" % (ex, eF, rx, rF))
    assert ex <= 1e-4 and eF <= 1e-4


def test_trajectory_sdf_terrain_small():
    """Drucker-Prager slab on a terrain SDF (64^3 version of the slope scene)."""
    sc = S.slope_flow(res=64, n_side=(50, 6, 50), dt=1e-4)
    eng = engine_for_scene(sc)
    eng.run_substeps(sc.params.dt, 60)
    gs = eng.state()
    mix = oracle_for(sc, "mixed")
    mix.run(60)
    ms = mix.get_state()
    ex, eF = rel_l2(gs["P"][:, :3], ms["P"][:, :3]), rel_l2(state_F(gs), state_F(ms))
    print("terrain 60 substeps: x %.3e F %.3e vs mixed" % (ex, eF))
    assert ex <= 1e-4 and eF <= 1e-4


# ----------------------------------------------------------------------------- engine surface
def test_engine_default_lattice_and_append():
    from nebula_b200.engine import MPMConfig, MPMEngine
    eng = MPMEngine(MPMConfig(nx=4, ny=3, nz=2, domainSize=(10, 10, 10), cellSize=10 / 64, maxParticles=30))
    assert eng.liveParticleCount() == 24
    P = eng.download("P")
    sp = 10 * 0.4 / 4
    assert np.allclose(P[0, :3], [5 - sp * 1.5, 7 - sp * 1.0, 5 - sp * 0.5], atol=1e-5)
    assert np.allclose(P[:, 3], sp ** 3)
    F0 = eng.download("F0")
    assert np.allclose(F0, [1, 0, 0, 0])
    pos = np.tile([[5.0, 5.0, 5.0, 0.1]], (10, 1)).astype(np.float32)
    vel = np.zeros((10, 4), np.float32)
    assert eng.appendParticles(pos, vel) == 6  # truncated at capacity
    assert eng.liveParticleCount() == 30
    eng.resetParticles()
    assert eng.liveParticleCount() == 0
    eng.step(1 / 60)  # no particles: a valid no-op


def test_engine_non_cube_domain_clamp():
    """8-1 (test_mpm.cpp:749-791): a flat 20x5x20 domain clamps the short axis."""
    from nebula_b200.engine import MPMConfig, MPMEngine
    cfg = MPMConfig(nx=0, ny=0, nz=0, maxParticles=4, domainSize=(20.0, 5.0, 20.0), cellSize=1.25)
    eng = MPMEngine(cfg)
    Vp = 1.25 ** 3
    eng.appendParticles(np.array([[10.0, 2.5, 10.0, Vp]], np.float32), np.array([[0.0, 50.0, 0.0, 0.0]], np.float32))
    for _ in range(30):
        eng.step(1 / 60)
    p = eng.download("P")[0]
    assert np.isfinite(p[1]) and p[1] <= 5.0 and p[1] > 5.0 * 0.3
    assert abs(p[0] - 10) < 2 and abs(p[2] - 10) < 2


def test_engine_errors_and_flags():
    from nebula_b200._capi import NebulaError
    from nebula_b200.engine import MPMConfig, MPMEngine
    eng = MPMEngine(MPMConfig(nx=2, ny=2, nz=2, domainSize=(1, 1, 1), cellSize=1 / 16))
    with pytest.raises(NebulaError):
        eng.setColliderSDF(np.zeros(10, np.float32))
    bad = np.zeros(1, S.FORCE_DTYPE)
    bad["type"] = 2  # turbulence
    with pytest.raises(NebulaError):
        eng.setForces([bad[0]])
    # a non-finite particle raises the device error flag, reported at sync
    st = eng.state()
    st["P"][0, 0] = np.nan
    eng.upload_state(st)
    eng.step(1e-3)
    with pytest.raises(NebulaError):
        eng.sync()
