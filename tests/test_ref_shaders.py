"""The CPU oracle against the reference's own MPM shaders, run on the CPU.

``oracle/build_ref.py`` compiles the reference's GLSL compute shaders
(shaders/mpm_*.comp with mpm_common / collider_common / force_common /
force_noise .glsl, and the force functions of src/core/Force.h) unchanged in
meaning for the CPU, and ``oracle/ref_dispatch.cpp`` issues them in the order
of MPMEngine::step.  These tests run that build and the oracle in its "ref32"
mode on the same seeded inputs and require the results to be identical bit
for bit: binning, P2G, grid update with forces / colliders / dense SDF, G2P
for every material model of the reference under APIC, PIC and FLIP (with the
J-reset and the SDF push-out taken), multi-substep trajectories, and the
PBF engine's spatial hash (hash_count.comp / hash_sort.comp).  They
pin the oracle -- the checker of every GPU parity test -- to the reference's
code itself.  They need no GPU; they are skipped only where neither the
reference tree nor an earlier build of the library is present.
"""
import numpy as np
import pytest

import oracle
from nebula_b200 import scenes as S
from oracle import ref as R

pytestmark = pytest.mark.skipif(not R.available(), reason="reference shader library absent (no reference tree, no earlier build)")

MODELS = [(S.MAT_ELASTIC, "elastic"), (S.MAT_VON_MISES, "von_mises"), (S.MAT_DRUCKER_PRAGER, "drucker_prager"),
          (S.MAT_GRANULAR_POWDER, "powder"), (S.MAT_FLUID, "fluid"), (S.MAT_VISCOPLASTIC_MUD, "mud")]
TRANSFERS = [(-1.0, "apic"), (0.0, "pic"), (0.7, "flip")]


def pair(sp, state, sdf=None, threads=1):
    o = oracle.Oracle("ref32")
    r = R.RefShaders(threads)
    for x in (o, r):
        x.set_params(sp)
        x.set_sdf(sdf)
        x.set_state(state)
    return o, r


def bits(a):
    return np.ascontiguousarray(np.asarray(a, np.float32)).view(np.uint32)


def assert_same_state(o, r, what=""):
    a, b = o.get_state(), r.get_state()
    for f in oracle.FIELDS:
        lanes = 3 if f == "v" else 4  # v.w carries the material id; the oracle keeps it apart
        same = bits(a[f][:, :lanes]) == bits(b[f][:, :lanes])
        assert same.all(), "%s %s: %d of %d values differ" % (what, f, (~same).sum(), same.size)
    assert np.array_equal(a["mat"], b["mat"])


def assert_same_grid(o, r, what=""):
    (mo, ma), (mr, mar) = o.get_grid(), r.get_grid()
    assert np.array_equal(bits(ma), bits(mar)), what + " grid mass"
    assert np.array_equal(bits(mo), bits(mr)), what + " grid momentum"


def ref_advanced(sc, n, sdf=None):
    """The scene's state after n substeps of the reference's shaders."""
    r = R.RefShaders(4)
    r.set_params(sc.params)
    r.set_sdf(sdf)
    r.set_state(sc.state)
    r.run(n)
    st = r.get_state()
    return {f: st[f] for f in oracle.FIELDS}


def sphere_sdf(res, centre, radius):
    """Morton-ordered SDF of a sphere (negative inside) at cell centres."""
    nc = S.hash_cells((res, res, res))
    c = (np.arange(res) + 0.5) / res
    X, Y, Z = np.meshgrid(c, c, c, indexing="ij")
    sdf = np.full(nc, 1e6, np.float32)
    codes = S.morton_encode(*np.meshgrid(np.arange(res), np.arange(res), np.arange(res), indexing="ij"))
    d = np.sqrt((X - centre[0]) ** 2 + (Y - centre[1]) ** 2 + (Z - centre[2]) ** 2) - radius
    sdf[codes.ravel()] = d.ravel().astype(np.float32)
    return sdf


# ----------------------------------------------------------------------------- binning
@pytest.mark.parametrize("res", [32, 64])
def test_bins_identical(res):
    """zero cells, hash count, the three scan passes and the hash sort; with
    particles outside the domain (clamped into the edge cells)."""
    sc = S.elastic_block(res=res)
    rng = np.random.default_rng(11)
    P = sc.state["P"]
    out = rng.random(P.shape[0]) < 0.02
    P[out, :3] = (rng.random((out.sum(), 3)) * 1.6 - 0.3).astype(np.float32)
    o, r = pair(sc.params, sc.state)
    for x in (o, r):
        x.zero_grid()
        x.bin()
    for a, b, name in zip(o.get_bins(), r.get_bins(), ("cellCount", "cellOffset", "sorted")):
        assert np.array_equal(a, b), name


def test_scan_beyond_1024_groups_is_not_a_prefix_in_the_reference():
    """On 128^3 (8,192 scan groups) the reference's single 1024-wide global scan
    leaves the groups from 1024 on with their own total as base: its offsets
    there are not the prefix sum, while the oracle (and the CUDA path) use the
    intended exclusive scan.  Counts agree everywhere, offsets below cell
    262,144 agree."""
    sc = S.multimaterial(res=128)
    o, r = pair(sc.params, sc.state)
    for x in (o, r):
        x.zero_grid()
        x.bin()
    (co, oo, _), (cr, orr, _) = o.get_bins(), r.get_bins()
    assert np.array_equal(co, cr)
    assert np.array_equal(oo, np.cumsum(co, dtype=np.uint64).astype(np.uint32))
    lim = 1024 * 256
    assert np.array_equal(oo[:lim], orr[:lim])
    occupied = np.nonzero(co[lim:])[0] + lim
    assert occupied.size > 0 and np.any(oo[occupied] != orr[occupied])


# ----------------------------------------------------------------------------- P2G
@pytest.mark.parametrize("flip,tname", TRANSFERS, ids=[t for _, t in TRANSFERS])
def test_p2g_identical(flip, tname):
    """The per-node gather over a state 10 substeps into the shear block
    (nonzero affine B and packed stress), two-material table."""
    sc = S.shear_block(S.MAT_VON_MISES, flip_ratio=flip)
    sc.params.materials = sc.params.materials + [S.preset_sand()]
    state = ref_advanced(sc, 10)
    state["v"][::3, 3] = np.uint32(1).view(np.float32)  # every third particle is material 1
    o, r = pair(sc.params, state)
    for x in (o, r):
        x.zero_grid()
        x.bin()
        x.p2g()
    assert_same_grid(o, r, "p2g")


# ----------------------------------------------------------------------------- grid update
def colliders():
    box = np.zeros(1, S.COLLIDER_DTYPE)
    box["type"], box["pos"], box["nrm"], box["vel"], box["restitution"], box["friction"] = 2, (0.2, 0.6, 0.3), (0.1, 0.05, 0.1), (0, 0.3, 0), 0.5, 0.1
    plane = np.zeros(1, S.COLLIDER_DTYPE)
    plane["type"], plane["pos"], plane["nrm"], plane["restitution"], plane["friction"] = 0, (0, 0.15, 0), (0.1, 1.0, 0.0), 0.0, 0.5
    cap = np.zeros(1, S.COLLIDER_DTYPE)
    cap["type"], cap["pos"], cap["nrm"], cap["radius"], cap["friction"] = 3, (0.7, 0.4, 0.2), (0.0, 0.3, 0.4), 0.06, 0.2
    return [S.sphere_collider((0.5, 0.3, 0.5), 0.15, vel=(0.1, 0.0, -0.2), restitution=0.2, friction=0.3), box[0], plane[0], cap[0]]


def test_grid_update_identical():
    """Momentum -> velocity, the 15 m/s cap, gravity and wind (one wind masked
    off for MPM), the wall band, all four analytic colliders (moving), the
    dense-SDF boundary; both halves of the momentum buffer."""
    sc = S.elastic_block()
    sp = sc.params
    sp.colliders = colliders()
    sp.forces = [S.gravity(), S.wind((0.3, 0.0, 1.0), 2.0, affect_mask=1), S.wind((1.0, 0.0, 0.0), 50.0, affect_mask=2)]
    nc = sp.hash_cells
    rng = np.random.default_rng(7)
    mass = np.where(rng.random(nc) < 0.3, rng.random(nc).astype(np.float32) * 1e-3, 0).astype(np.float32)
    mass[rng.random(nc) < 0.01] = 5e-11
    mom = np.zeros((2 * nc, 4), np.float32)
    mom[:nc, :3] = (rng.standard_normal((nc, 3)) * 2e-3).astype(np.float32)
    mom[:nc][rng.random(nc) < 0.01, :3] *= 1e4
    sdf = sphere_sdf(64, (0.6, 0.2, 0.5), 0.2)
    o, r = pair(sp, sc.state, sdf)
    for x in (o, r):
        x.set_grid(mom, mass)
        x.grid_update()
    assert_same_grid(o, r, "grid update")
    for x in (o, r):
        x.sdf_bc()
    assert_same_grid(o, r, "sdf boundary")


# ----------------------------------------------------------------------------- G2P
@pytest.mark.parametrize("flip,tname", TRANSFERS, ids=[t for _, t in TRANSFERS])
@pytest.mark.parametrize("model,mname", MODELS, ids=[m for _, m in MODELS])
def test_substep_pass_by_pass_identical(model, mname, flip, tname):
    """One substep pass by pass from a state 15 substeps into the shear block:
    the grid after P2G, grid update and SDF boundary, then every particle
    field after G2P (F, the packed Kirchhoff stress, B, x, v).  2% of the
    particles get |det F| outside [0.15, 10] (the J-reset), and a sphere SDF
    holds part of the block (the particle push-out)."""
    sc = S.shear_block(model, flip_ratio=flip)
    state = ref_advanced(sc, 15)
    rng = np.random.default_rng(model * 10 + int(flip * 10) + 10)
    n = state["P"].shape[0]
    pick = rng.random(n) < 0.02
    scale = np.where(rng.random(n) < 0.5, 2.5, 0.45).astype(np.float32)
    for f in ("F0", "F1", "F2"):
        state[f][pick, :3] *= scale[pick, None]
    sdf = sphere_sdf(64, (0.5, 0.55, 0.5), 0.08)
    o, r = pair(sc.params, state, sdf)
    for step in ("zero_grid", "bin", "p2g", "grid_update", "sdf_bc"):
        for x in (o, r):
            getattr(x, step)()
    assert_same_grid(o, r, mname + " " + tname)
    for x in (o, r):
        x.g2p()
    assert_same_state(o, r, mname + " " + tname)


@pytest.mark.parametrize("key,nsub", [("cfg2", 20), ("cfg3", 3)], ids=["cfg2_multimaterial_80k_128", "cfg3_slope_1m_256"])
def test_configurations_above_1024_scan_groups_with_the_intended_scan(key, nsub):
    """The two-material scene on 128^3 and the benched slope (1M particles on
    256^3 over the terrain SDF) through every compiled shader, with the scan
    passes giving the exclusive prefix they intend: identical to the oracle
    bit for bit, so at these sizes the oracle differs from the reference's
    shaders only by the scan's 1024-group limit."""
    sc = S.load_config(key)
    o = oracle.Oracle("ref32")
    r = R.RefShaders(8, intended_scan=True)
    for x in (o, r):
        x.set_params(sc.params)
        x.set_sdf(sc.sdf)
        x.set_state(sc.state)
    o.run(nsub)
    r.run(nsub)
    assert_same_state(o, r, key)


# ----------------------------------------------------------------------------- edge cases
def test_empty_scene_identical():
    """No particles: every pass runs over an empty set and leaves an empty grid."""
    sc = S.elastic_block()
    empty = {f: np.zeros((0, 4), np.float32) for f in oracle.FIELDS}
    o, r = pair(sc.params, empty)
    for x in (o, r):
        x.run(2)
    assert_same_grid(o, r, "empty")
    for a, b in zip(o.get_bins(), r.get_bins()):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("model,mname", MODELS, ids=[m for _, m in MODELS])
def test_global_parameters_without_a_material_table(model, mname):
    """materialCount 0: P2G takes rho0 and G2P takes mu, lambda, the plastic
    model, M, q_c and q_max from the push constants (mpm_g2p.comp:139-149,
    mpm_p2g.comp:50-55); bulkK and the viscosity are then 0."""
    sc = S.shear_block(model)
    sp = sc.params
    sp.materials = []
    sp.plastic_model = model
    sp.mu_lame, sp.lambda_lame = S.lame(3e4, 0.3)
    sp.M_friction, sp.q_cohesion, sp.q_max = 0.6, 5.0, 150.0
    sp.rho0 = 1200.0
    o, r = pair(sp, sc.state)
    o.run(12)
    r.run(12)
    assert_same_state(o, r, "global " + mname)


def test_material_ids_past_the_table_are_clamped():
    """Ids at and past the table's end read its last entry (min(id, count - 1))."""
    sc = S.shear_block(S.MAT_ELASTIC)
    sc.params.materials = sc.params.materials + [S.preset_mud()]
    ids = np.arange(sc.state["P"].shape[0], dtype=np.uint32) % 5  # 0..4 over a table of 2
    sc.state["v"][:, 3] = ids.view(np.float32)
    o, r = pair(sc.params, sc.state)
    o.run(10)
    r.run(10)
    assert_same_state(o, r, "clamped ids")


def test_walls_and_world_clamp_identical():
    """Particles in the two-node wall band of all six faces and past the
    1.5-cell margin, moving outward: the grid's wall band and G2P's world
    clamp (mpm_grid_update.comp:54-60, mpm_g2p.comp:255-263)."""
    sc = S.shear_block(S.MAT_DRUCKER_PRAGER)
    rng = np.random.default_rng(5)
    n = sc.state["P"].shape[0]
    P, v = sc.state["P"], sc.state["v"]
    face = rng.integers(0, 6, n)
    axis, side = face // 2, face % 2
    depth = rng.uniform(-0.02, 0.04, n).astype(np.float32)  # some past the domain
    P[np.arange(n), axis] = np.where(side == 0, depth, 1.0 - depth).astype(np.float32)
    v[np.arange(n), axis] = np.where(side == 0, -3.0, 3.0).astype(np.float32)
    o, r = pair(sc.params, sc.state)
    o.run(8)
    r.run(8)
    assert_same_state(o, r, "walls")


# ----------------------------------------------------------------------------- PBF spatial hash
def test_pbf_hash_identical():
    """The PBF engine's spatial hash (hash_count.comp, the scan passes,
    hash_sort.comp) against the oracle that checks nebula_hash_bin: a
    hand-worked case, the fluid layout with its unused slots (type flag 6),
    and a non-cubic offset grid with particles outside it.  Bit-exact."""
    from nebula_b200 import hash as H
    hand = np.array([[0.5, 0.5, 0.5, 1], [1.5, 0.2, 0.1, 1], [0.1, 1.9, 0.0, 1], [1.2, 1.2, 1.2, 1], [0.3, 0.3, 0.3, 0],
                     [-5.0, 9.0, 0.7, 1], [0.9, 0.1, 0.2, 1], [5.0, 5.0, 5.0, 1]], np.float32)
    cases = [(hand, np.array([0, 0, 3, 0, 6, 0, 3, 0], np.uint32), (0, 0, 0), 1.0, (2, 2, 2), 8)]
    p, f = H.fluid_layout()
    g = H.FluidGrid()
    cases.append((p, f, g.world_min, g.cell_size, g.grid_res, g.hash_cells))
    rng = np.random.default_rng(3)
    g = H.FluidGrid(domain_size=(3.0, 1.0, 2.0), cell_size=0.05, world_min=(-1.0, 0.5, 2.0))
    q = np.zeros((20000, 4), np.float32)
    q[:, :3] = rng.uniform(-0.2, 1.2, (20000, 3)) * np.array(g.domain_size) + np.array(g.world_min)
    cases.append((q, None, g.world_min, g.cell_size, g.grid_res, g.hash_cells))
    for args in cases:
        for a, b, name in zip(oracle.hash_bin(*args), R.hash_bin(*args), ("cellCount", "cellOffset", "sortedIdx")):
            assert np.array_equal(a, b), name


# ----------------------------------------------------------------------------- trajectories
def slope_small():
    return S.slope_flow(res=64, n_side=(60, 6, 60), substeps=40, dt=1e-4, lift=-1.0)


@pytest.mark.parametrize("make,nsub", [(lambda: S.elastic_block(), 25),
                                       (lambda: S.shear_block(S.MAT_DRUCKER_PRAGER, flip_ratio=0.7), 25),
                                       (lambda: S.multimaterial(res=64, dt=1e-4), 20),
                                       (slope_small, 40)],
                         ids=["elastic_block", "shear_dp_flip", "multimaterial_64", "slope_terrain_64"])
def test_trajectory_identical(make, nsub):
    sc = make()
    o, r = pair(sc.params, sc.state, sc.sdf)
    o.run(nsub)
    r.run(nsub)
    assert_same_state(o, r, sc.name)


def test_threaded_dispatch_identical():
    """The CPU arm of the benchmark spreads the independent per-invocation
    passes over threads; that changes no result."""
    sc = S.multimaterial(res=64, dt=1e-4)
    a, b = R.RefShaders(1), R.RefShaders(8)
    for x in (a, b):
        x.set_params(sc.params)
        x.set_sdf(None)
        x.set_state(sc.state)
        x.run(5)
    sa, sb = a.get_state(), b.get_state()
    for f in oracle.FIELDS:
        assert np.array_equal(bits(sa[f]), bits(sb[f])), f


def test_a_planted_change_in_the_oracle_is_seen():
    """The comparison is not vacuous: the oracle with dt one part in 1e6 off
    differs from the reference after one substep."""
    sc = S.shear_block(S.MAT_DRUCKER_PRAGER)
    o, r = pair(sc.params, sc.state)
    p = oracle.make_params(sc.params)
    p.dt = np.float32(sc.params.dt * (1 + 1e-6))
    o._L.orc_set_params(o._h, oracle.C.byref(p))
    o.run(1)
    r.run(1)
    with pytest.raises(AssertionError):
        assert_same_state(o, r, "planted")
