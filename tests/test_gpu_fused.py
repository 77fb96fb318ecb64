"""The brick-sparse fused pipeline (default engine path) on the GPU.

Checks the engine's own brick binning against the oracle's cell binning, the
fused pipeline against the dense one and the oracle, and the host paths that
invalidate a pending P2G (dt changes, uploads, appends, parameter changes).
"""
import numpy as np
import pytest

from nebula_b200 import scenes as S
from nebula_b200.engine import engine_for_scene

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def oracle_run(sc, n, mode="ref32"):
    from oracle import Oracle
    o = Oracle(mode)
    o.set_params(sc.params)
    o.set_sdf(sc.sdf)
    o.set_state(sc.state)
    o.run(n)
    return o.get_state()


def Fm(st):
    return np.concatenate([st["F0"][:, :3], st["F1"][:, :3], st["F2"][:, :3]], axis=1)


@pytest.mark.parametrize("make", [S.elastic_block, S.multimaterial, lambda: S.slope_flow(with_sdf=False)],
                         ids=["elastic_8k_64", "multimaterial_80k_128", "slope_1m_256"])
def test_brick_bins_match_oracle_cells(make):
    """Every listed brick holds exactly the particles whose cell Morton code >> 6
    is that brick; bricks are listed in ascending order."""
    sc = make()
    eng = engine_for_scene(sc)
    ids, starts, pids = eng.export_brick_bins()
    from oracle import Oracle
    o = Oracle("ref32")
    o.set_params(sc.params)
    o.set_state(sc.state)
    o.bin()
    cnt, off, srt = o.get_bins()
    cell_of = np.empty(sc.n, np.uint32)
    nz = np.nonzero(cnt)[0]
    for c in nz:
        cell_of[srt[off[c] - cnt[c]:off[c]]] = c
    brick_of = cell_of >> 6
    assert np.all(np.diff(ids.astype(np.int64)) > 0)
    assert starts[0] == 0 and starts[-1] == sc.n
    assert np.array_equal(np.sort(pids), np.arange(sc.n, dtype=np.uint32))
    seg = np.repeat(ids, np.diff(starts))
    assert np.array_equal(seg, brick_of[pids])


def test_brick_bins_after_substeps():
    """Binning produced inside the fused kernel after 30 substeps: bricks in
    ascending order, the particles of a brick in cell order."""
    sc = S.shear_block()
    eng = engine_for_scene(sc)
    eng.run_substeps(sc.params.dt, 30)
    st = eng.state()
    ids, starts, pids = eng.export_brick_bins()
    h = sc.params.cell_size
    g = np.clip(np.floor(st["P"][:, :3].astype(np.float32) / np.float32(h)), 0, 63).astype(np.int64)
    cell = S.morton_encode(g[:, 0], g[:, 1], g[:, 2])
    brick = cell >> 6
    assert np.array_equal(np.repeat(ids, np.diff(starts)), brick[pids])
    # inside a brick the particles are in cell order
    assert np.all(np.diff(cell[pids].astype(np.int64)) >= 0)


@pytest.mark.parametrize("make,n", [(S.shear_block, 100), (S.multimaterial, 60)], ids=["elastic_shear", "multimaterial"])
def test_fused_matches_dense(make, n):
    sc = make()
    a = engine_for_scene(sc, pipeline="fused")
    b = engine_for_scene(sc, pipeline="dense")
    a.run_substeps(sc.params.dt, n)
    b.run_substeps(sc.params.dt, n)
    sa, sb = a.state(), b.state()
    ex, ev = rel_l2(sa["P"][:, :3], sb["P"][:, :3]), rel_l2(sa["v"][:, :3], sb["v"][:, :3])
    print("fused vs dense after %d substeps: x %.2e v %.2e" % (n, ex, ev))
    assert ex < 1e-5 and ev < 1e-3


def test_fused_elastic_shear_vs_oracle_in_chunks():
    """100 substeps as 7 step() calls of different dt lengths (pending grid
    rebuilt whenever the substep length changes)."""
    sc = S.shear_block()
    eng = engine_for_scene(sc)
    dt = sc.params.dt
    for k in (10, 20, 5, 25, 15, 10, 15):
        eng.run_substeps(dt, k)
    gs = eng.state()
    rs = oracle_run(sc, 100)
    ex, eF = rel_l2(gs["P"][:, :3], rs["P"][:, :3]), rel_l2(Fm(gs), Fm(rs))
    print("chunked fused: x %.2e F %.2e" % (ex, eF))
    assert ex <= 1e-4 and eF <= 1e-4


def test_fused_dt_change_rebuilds_pending_grid():
    sc = S.shear_block()
    eng = engine_for_scene(sc)
    dt = sc.params.dt
    eng.run_substeps(dt, 10)
    eng.run_substeps(dt / 2, 10)  # different substep length
    gs = eng.state()
    from oracle import Oracle
    o = Oracle("ref32")
    o.set_params(sc.params)
    o.set_state(sc.state)
    o.run(10)
    sp2 = sc.params
    sp2.dt = dt / 2
    o.set_params(sp2)
    o.run(10)
    rs = o.get_state()
    assert rel_l2(gs["P"][:, :3], rs["P"][:, :3]) < 1e-5
    assert rel_l2(Fm(gs), Fm(rs)) < 1e-5


def test_fused_host_edits_between_steps():
    """Upload / append / material ids between steps see particles in original order."""
    sc = S.shear_block()
    eng = engine_for_scene(sc, capacity=sc.n + 100)
    eng.run_substeps(sc.params.dt, 10)
    st = eng.state()
    # original order after reordering: particle 0 is still particle 0
    rs = oracle_run(sc, 10)
    assert rel_l2(st["P"][:, :3], rs["P"][:, :3]) < 1e-6
    # append 100 particles and keep stepping
    pos = np.tile(np.array([[0.3, 0.3, 0.3, 1e-6]], np.float32), (100, 1))
    pos[:, 0] += np.linspace(0, 0.05, 100, dtype=np.float32)
    vel = np.zeros((100, 4), np.float32)
    assert eng.appendParticles(pos, vel) == 100
    eng.run_substeps(sc.params.dt, 10)
    st2 = eng.state()
    assert st2["P"].shape[0] == sc.n + 100
    assert np.all(np.isfinite(st2["P"]))
    # the appended particles fell under gravity only
    assert np.all(st2["v"][sc.n:, 1] < 0)
    # re-upload the original scene: result equals a fresh run
    eng.upload_state(sc.state)
    eng.run_substeps(sc.params.dt, 10)
    st3 = eng.state()
    assert rel_l2(st3["P"][:, :3], rs["P"][:, :3]) < 1e-6


def test_fused_flip_and_pic_vs_oracle():
    for flip in (0.0, 0.95):
        sc = S.shear_block(flip_ratio=flip)
        eng = engine_for_scene(sc)
        eng.run_substeps(sc.params.dt, 60)
        gs = eng.state()
        rs = oracle_run(sc, 60)
        ex, ev = rel_l2(gs["P"][:, :3], rs["P"][:, :3]), rel_l2(gs["v"][:, :3], rs["v"][:, :3])
        print("flip %.2f: x %.2e v %.2e" % (flip, ex, ev))
        assert ex < 1e-5 and ev < 1e-4


def test_fused_fast_particle_leaves_tile():
    """A FLIP particle crossing several cells per substep scatters outside its
    block tile (global-reduction path) and still matches the oracle."""
    sp = S.StepParams(dt=5e-3, cell_size=1.0 / 16, domain_size=(1.0, 1.0, 1.0), flip_ratio=1.0,
                      materials=[S.material(S.MAT_ELASTIC, 1e3, 0.3, 1000.0)], forces=[])
    pos = np.array([[0.3, 0.5, 0.5], [0.5, 0.5, 0.5]], np.float32)
    st = S.make_state(pos, np.float32(1e-4), vel=np.array([[40.0, 0.0, 0.0], [0.0, 0.0, 0.0]], np.float32))
    sc = S.Scene("fast", sp, st, 8)
    eng = engine_for_scene(sc)
    eng.run_substeps(sp.dt, 4)
    gs = eng.state()
    assert eng.stats()["overflow_particles"] > 0
    rs = oracle_run(sc, 4)
    assert rel_l2(gs["P"][:, :3], rs["P"][:, :3]) < 1e-6
    assert rel_l2(gs["v"][:, :3], rs["v"][:, :3]) < 1e-5


def test_fused_export_grid_after_step_is_p2g_of_state():
    """The grid left pending by the fused kernel equals a fresh P2G of the
    updated particles."""
    sc = S.shear_block()
    eng = engine_for_scene(sc)
    eng.run_substeps(sc.params.dt, 12)
    mom, mass = eng.export_grid(sc.params.dt)  # pending grid from the fused scatter
    st = eng.state()
    sc2 = S.Scene("x", sc.params, st, 0)
    fresh = engine_for_scene(sc2)
    fmom, fmass = fresh.export_grid(sc.params.dt)  # standalone P2G
    assert rel_l2(mom[:, :3], fmom[:, :3]) < 1e-5 and rel_l2(mass, fmass) < 1e-5


def test_downloads_follow_every_state_change():
    """The original-order copy behind downloads is rebuilt once per state
    version: after each step, upload, material-id edit and reset the fields
    read back are the current ones."""
    sc = S.shear_block()
    dt = sc.params.dt
    a, b = engine_for_scene(sc), engine_for_scene(sc)
    a.run_substeps(dt, 5)
    p1, v1 = a.download("P"), a.download("v")
    assert np.array_equal(a.download("P"), p1)  # same version: same copy
    a.run_substeps(dt, 5)
    p2 = a.download("P")
    b.run_substeps(dt, 10)
    pb = b.download("P")
    assert np.abs(p2[:, :3] - p1[:, :3]).max() > 1e-5
    assert np.linalg.norm(p2 - pb) / np.linalg.norm(pb) < 1e-6
    a.setParticleMaterialIds(np.zeros(sc.n, np.uint32))
    assert not a.download("v")[:, :3].any()  # the reference zeroes v with the ids
    a.upload_state(sc.state)
    assert np.array_equal(a.download("P"), sc.state["P"]) and np.array_equal(a.download("v"), sc.state["v"])
    a.run_substeps(dt, 3)
    a.resetParticles()
    assert a.liveParticleCount() == 0


def test_fused_matches_dense_on_a_512_grid():
    """A 512^3 grid (134,217,728 hash cells, 2,097,152 bricks): particle
    blocks at the domain's corners, one moving into the top wall band, through
    both pipelines."""
    h = 1.0 / 512
    sp = 0.5 * h
    blocks = []
    for k, origin in enumerate(((0.01, 0.01, 0.01), (0.93, 0.97, 0.94), (0.48, 0.5, 0.47))):
        blocks.append(S.jittered_lattice(9, k, (24, 24, 24), sp, origin, 0.25 * h))
    pos = np.concatenate(blocks)
    vel = np.zeros_like(pos)
    vel[len(blocks[0]):2 * len(blocks[0]), 1] = 2.0  # towards the top wall band
    mats = [S.material(S.MAT_ELASTIC, 1e4, 0.3, 1000.0)]
    params = S.StepParams(dt=2e-5, cell_size=float(np.float32(h)), domain_size=(1.0, 1.0, 1.0), flip_ratio=-1.0, materials=mats,
                          forces=[S.gravity()])
    sc = S.Scene("corners_41k_512", params, S.make_state(pos, np.float32(sp) ** 3, vel=vel), 20)
    assert sc.params.hash_cells == 512 ** 3
    a = engine_for_scene(sc, pipeline="fused")
    b = engine_for_scene(sc, pipeline="dense")
    a.run_substeps(sc.params.dt, 20)
    b.run_substeps(sc.params.dt, 20)
    sa, sb = a.state(), b.state()
    a.cleanup()
    b.cleanup()
    assert rel_l2(sa["P"][:, :3], sb["P"][:, :3]) < 1e-6
    assert rel_l2(sa["v"][:, :3], sb["v"][:, :3]) < 1e-4
    assert np.all(np.isfinite(sa["P"])) and sa["P"][:, 1].max() <= 1.0 - 1.5 * h + 1e-6  # the G2P clamp


def test_device_pointer_and_set_gravity():
    """nebula_mpm_device_ptr gives the fields in the original particle order
    after a step, and a write through it is seen by the next step;
    nebula_mpm_set_gravity replaces only the gravity entry of the table."""
    import ctypes as C

    from cuda.bindings import runtime as rt

    from nebula_b200 import _capi
    sc = S.shear_block()
    dt = sc.params.dt
    a = engine_for_scene(sc)
    a.run_substeps(dt, 7)
    n = a.liveParticleCount()
    host = np.empty((n, 4), np.float32)
    for f in ("P", "v", "F1"):
        ptr = a.device_ptr(f)
        (err,) = rt.cudaMemcpy(host.ctypes.data, ptr, host.nbytes, rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)
        assert err == rt.cudaError_t.cudaSuccess
        assert np.array_equal(host, a.download(f)), f
    # zero every velocity through the pointer; compare with an engine given the same state from the host
    st = a.state()
    (err,) = rt.cudaMemset(a.device_ptr("v"), 0, n * 16)
    assert err == rt.cudaError_t.cudaSuccess
    st["v"][:] = 0.0
    b = engine_for_scene(sc)
    b.upload_state(st)
    a.run_substeps(dt, 5)
    b.run_substeps(dt, 5)
    assert rel_l2(a.download("P")[:, :3], b.download("P")[:, :3]) < 1e-6
    # gravity through the C ABI, a wind kept: same as setting the table directly
    c, d = engine_for_scene(sc), engine_for_scene(sc)
    c.setForces([S.gravity(), S.wind((1.0, 0.0, 0.0), 2.0)])
    _capi.call("nebula_mpm_set_gravity", c._h, C.c_float(0.0), C.c_float(-3.0), C.c_float(1.0))
    d.setForces([S.wind((1.0, 0.0, 0.0), 2.0), S.gravity((0.0, -3.0, 1.0))])
    c.run_substeps(dt, 10)
    d.run_substeps(dt, 10)
    assert rel_l2(c.download("v")[:, :3], d.download("v")[:, :3]) < 1e-6


def test_step_is_graph_capturable():
    """nebula_mpm_step captured into a CUDA graph (torch.cuda.graph) and
    replayed advances the state like eager steps on the same stream, with an
    even number of substeps (the ping-pong state buffers end every step in the
    parity the graph was captured with)."""
    import torch

    sc = S.shear_block()
    dt = sc.params.dt
    a, b = engine_for_scene(sc), engine_for_scene(sc)
    for e in (a, b):
        e.numSubsteps = 6
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        a.step(dt * 6, s)  # first step outside capture: binning + pending grid, launch shapes resolved
        a.sync()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            a.step(dt * 6, s)
        for _ in range(4):
            g.replay()
        torch.cuda.synchronize()
    # capture only records: a ran 1 eager step + 4 replays
    b.step(dt * 6, s)
    for _ in range(4):
        b.step(dt * 6, s)
    b.sync()
    pa, pb = a.download("P")[:, :3], b.download("P")[:, :3]
    assert rel_l2(pa, pb) < 1e-6


def test_engines_on_concurrent_host_threads():
    """Four engines created and stepped from four host threads at once, each
    on its own stream (the library keeps no per-process mutable state beyond
    the once-per-device launch shapes): each equals a sequential run."""
    import threading

    import torch

    sc = S.shear_block()
    dt = sc.params.dt
    ref = engine_for_scene(sc)
    ref.run_substeps(dt, 20)
    want = ref.download("P")[:, :3]
    out, errors = [None] * 4, []

    def work(k):
        try:
            s = torch.cuda.Stream()
            e = engine_for_scene(sc)
            e.run_substeps(dt, 20, s)
            e.sync()
            out[k] = e.download("P")[:, :3]
            e.cleanup()
        except Exception as ex:  # reported below, on the main thread
            errors.append(ex)

    threads = [threading.Thread(target=work, args=(k,)) for k in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=120)
    assert not errors, errors
    for got in out:
        assert got is not None and rel_l2(got, want) < 1e-6
