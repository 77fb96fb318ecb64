"""Streaming state exchange (nebula_mpm_upload_state_async /
download_state_async / wait_downloads): a pipelined loop in which step k's
result is downloaded and step k + 1's input uploaded while step k computes
gives the same states as the synchronous upload / step / download, also when
the particle count changes between uploads."""
import numpy as np
import pytest

from nebula_b200 import _capi
from nebula_b200 import scenes as S
from nebula_b200.engine import engine_for_scene

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def pinned_like(state, n=None):
    import torch
    out = {}
    for f, a in state.items():
        m = a.shape[0] if n is None else n
        t = torch.empty((m, 4), dtype=torch.float32, pin_memory=True).numpy()
        t[:] = a[:m]
        out[f] = t
    return out


def inputs(sc):
    """Three different initial states of the shear block: the scene's own, a
    faster shear, and the first 6,000 particles with a vertical kick."""
    a = {f: v.copy() for f, v in sc.state.items()}
    b = {f: v.copy() for f, v in sc.state.items()}
    b["v"][:, 0] *= 1.5
    c = {f: v[:6000].copy() for f, v in sc.state.items()}
    c["v"][:, 1] += 0.5
    return [a, b, c]


@pytest.mark.parametrize("side_stream", [False, True], ids=["null_stream", "side_stream"])
def test_pipelined_exchange_equals_synchronous(side_stream):
    import torch

    sc = S.shear_block()
    dt = sc.params.dt
    states = inputs(sc)
    # synchronous reference: upload, 10 substeps, download
    ref = []
    b = engine_for_scene(sc)
    b.numSubsteps = 10
    for st in states:
        b.upload_state(st)
        b.step(dt * 10)
        ref.append(b.state())
    # pipelined through the async calls
    a = engine_for_scene(sc)
    a.numSubsteps = 10
    s = torch.cuda.Stream() if side_stream else None
    ins = [pinned_like(st) for st in states]
    outs = [pinned_like({f: np.zeros_like(v) for f, v in st.items()}) for st in states]
    a.upload_state_async(ins[0], s)
    for k in range(len(states)):
        a.step(dt * 10, s)
        a.download_state_async(outs[k], s)
        if k + 1 < len(states):
            a.upload_state_async(ins[k + 1], s)
    a.sync()
    assert a.liveParticleCount() == 6000
    for k, (got, want) in enumerate(zip(outs, ref)):
        for f in ("P", "v", "F0", "F1", "F2"):
            assert got[f].shape == want[f].shape
            assert rel_l2(got[f][:, :3], want[f][:, :3]) < 1e-5, (k, f)
    # wait_downloads orders a stream after the transfers
    if side_stream:
        a.step(dt * 10, s)
        last = pinned_like({f: np.zeros((6000, 4), np.float32) for f in sc.state})
        a.download_state_async(last, s)
        a.wait_downloads(s)
        s.synchronize()
        b.step(dt * 10)
        assert rel_l2(last["P"][:, :3], b.download("P")[:, :3]) < 1e-5


def test_async_calls_check_their_arguments():
    sc = S.shear_block()
    e = engine_for_scene(sc)
    with pytest.raises(ValueError):
        e.download_state_async({f: np.zeros((10, 4), np.float32) for f in sc.state})
    big = {f: np.zeros((sc.n + 1, 4), np.float32) for f in sc.state}
    with pytest.raises(_capi.NebulaError):
        e.upload_state_async(big)
    # the engine is still usable afterwards
    e.numSubsteps = 2
    e.step(sc.params.dt * 2)
    e.sync()
    assert e.liveParticleCount() == sc.n
