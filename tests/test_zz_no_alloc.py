"""nebula_mpm_bin_noalloc: binning with library-held scratch instead of a
caller workspace.  It runs the same kernels as nebula_mpm_bin, so on the same
positions its counts, range ends and sorted indices are identical.  The file
name sorts last so the GPU case also runs after every other test."""
import ctypes as C

import numpy as np
import pytest
import torch

from nebula_b200 import _capi, scenes as S
from nebula_b200.passes import PassRunner, make_pass


def _noalloc_bins(runner: PassRunner):
    """Bin runner.state[0] with nebula_mpm_bin_noalloc into fresh outputs."""
    dev = runner.dev
    cnt = torch.full((runner.nc,), -1, dtype=torch.int32, device=dev)
    off = torch.full((runner.nc,), -1, dtype=torch.int32, device=dev)
    srt = torch.full((max(runner.n, 1),), -1, dtype=torch.int32, device=dev)
    p = make_pass(runner.sp, runner.n)
    stream = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    _capi.call("nebula_mpm_bin_noalloc", C.byref(p), C.c_void_p(runner.state[0].data_ptr()), C.c_void_p(cnt.data_ptr()),
               C.c_void_p(off.data_ptr()), C.c_void_p(srt.data_ptr()), stream)
    torch.cuda.synchronize(dev)
    return (cnt.cpu().numpy().view(np.uint32), off.cpu().numpy().view(np.uint32), srt[: runner.n].cpu().numpy().view(np.uint32))


def test_noalloc_limits_and_rejection():
    """Sizes beyond the fixed scratch are refused before any device work."""
    lib = _capi.lib()
    assert lib.nebula_mpm_bin_noalloc_max_cells() == 128 ** 3
    assert lib.nebula_mpm_bin_noalloc_max_particles() == 1 << 18
    sp = S.slope_flow(with_sdf=False).params  # 256^3 cells
    p = make_pass(sp, 1000)
    rc = lib.nebula_mpm_bin_noalloc(C.byref(p), None, None, None, None, None)
    assert rc == _capi.ERR_INVALID
    assert b"exceeds the fixed maximum" in lib.nebula_mpm_last_error()
    sp = S.elastic_block().params  # 64^3 cells, within limits
    p = make_pass(sp, (1 << 18) + 1)
    rc = lib.nebula_mpm_bin_noalloc(C.byref(p), None, None, None, None, None)
    assert rc == _capi.ERR_INVALID
    assert b"particleCount" in lib.nebula_mpm_last_error()


@pytest.mark.gpu
def test_noalloc_matches_workspace_bin_two_calls(cuda_lib):
    """Two calls in a row on different scenes and grids (64^3 then 128^3),
    each identical to nebula_mpm_bin on the same positions."""
    runners = []
    for make in (S.elastic_block, S.multimaterial):
        sc = make()
        r = PassRunner(sc.params, sc.n)
        r.upload_particles(sc.state)
        runners.append(r)
    got = [_noalloc_bins(r) for r in runners]  # two calls in a row
    for r, g in zip(runners, got):
        r.bin()
        want = r.read_bins()
        for a, b in zip(g, want):
            assert np.array_equal(a, b)
        assert int(g[0].sum()) == r.n


@pytest.mark.gpu
def test_noalloc_status_reports_an_expired_wait(cuda_lib):
    """The error word of the library-held scratch reaches the caller through
    nebula_mpm_bin_noalloc_status: clean after a call, the scan-timeout bit
    after the probe has made the scan's bounded look-back expire, clean again
    after the next call, whose bins equal nebula_mpm_bin's."""
    lib = _capi.lib()
    sc = S.elastic_block()
    r = PassRunner(sc.params, sc.n)
    r.upload_particles(sc.state)
    stream = C.c_void_p(torch.cuda.current_stream(r.dev).cuda_stream)
    bits = C.c_uint32(7)
    first = _noalloc_bins(r)
    assert lib.nebula_mpm_bin_noalloc_status(C.byref(bits), stream) == _capi.OK and bits.value == 0
    p = make_pass(r.sp, r.n)
    counts = torch.zeros(r.nc, dtype=torch.int32, device=r.dev)  # the probe reads hashCells counts
    _capi.call("nebula_mpm_bin_noalloc_probe_wait_expiry", C.byref(p), C.c_void_p(counts.data_ptr()), stream)
    assert lib.nebula_mpm_bin_noalloc_status(C.byref(bits), stream) == _capi.ERR_DEVICE
    assert bits.value & 1, bits.value
    again = _noalloc_bins(r)
    assert lib.nebula_mpm_bin_noalloc_status(C.byref(bits), stream) == _capi.OK and bits.value == 0
    r.bin()
    for a, b, c in zip(again, first, r.read_bins()):
        assert np.array_equal(a, b) and np.array_equal(a, c)
