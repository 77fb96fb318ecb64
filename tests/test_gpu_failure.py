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
