"""Failure detection without a GPU fault: every wait in the kernels is
bounded.  A probe makes the brick scan's look-back wait on a predecessor that
never publishes; the kernel must give up, report the scan-timeout bit and
return, and the context must stay usable for the engine."""
import ctypes as C
import time

import numpy as np
import pytest

from nebula_b200 import _capi
from nebula_b200 import scenes as S
from nebula_b200.engine import engine_for_scene
from nebula_b200.passes import PassRunner

pytestmark = pytest.mark.gpu


def test_bounded_wait_expires_and_the_context_survives():
    bits = C.c_uint32(0)
    t0 = time.time()
    _capi.call("nebula_mpm_probe_wait_expiry", C.byref(bits))
    waited = time.time() - t0
    assert bits.value & 1, bits.value  # kErrScanTimeout
    assert waited < 30.0
    sc = S.shear_block()
    e = engine_for_scene(sc)
    e.run_substeps(sc.params.dt, 5)
    assert np.all(np.isfinite(e.download("P")))
    assert e.stats()["error_flags"] == 0


def test_binning_wait_expiry_reaches_the_caller():
    """The single-pass binning's scan waits are bounded too, and what they
    report reaches the caller through nebula_mpm_bin_status: clean after a
    normal call, the scan-timeout bit after the probe, clean again after the
    next call, whose bins are still the workspace binning's."""
    sc = S.elastic_block()
    r = PassRunner(sc.params, sc.n)
    r.upload_particles(sc.state)
    r.bin()
    assert r.bin_status() == (_capi.OK, 0)
    want = r.read_bins()
    t0 = time.time()
    r.probe_bin_wait_expiry()
    rc, bits = r.bin_status()
    assert time.time() - t0 < 30.0
    assert rc == _capi.ERR_DEVICE and bits & 1, (rc, bits)
    assert b"scan look-back wait expired" in _capi.lib().nebula_mpm_last_error()
    r.bin()
    assert r.bin_status() == (_capi.OK, 0)
    for a, b in zip(r.read_bins(), want):
        assert np.array_equal(a, b)
