import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))
TESTS = Path(__file__).resolve().parent
if str(TESTS) not in sys.path:
    sys.path.insert(0, str(TESTS))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the sm_100a kernels")
    config.addinivalue_line("markers", "slow: long-running parity case")


@pytest.fixture(scope="session", autouse=True)
def _built_oracle():
    """Build the CPU oracle once per session (test infrastructure)."""
    import oracle
    oracle.build()
    yield


@pytest.fixture(scope="session")
def cuda_lib():
    """The CUDA library, built in-tree, on a CUDA device.  A GPU test never
    skips silently: without a device or the library it fails."""
    import torch
    from nebula_b200 import build as nb
    nb.build()
    if not torch.cuda.is_available():
        pytest.fail("GPU test selected but torch.cuda.is_available() is False")
    from nebula_b200 import _capi
    return _capi.lib()


@pytest.fixture(autouse=True)
def _gpu_guard(request):
    if request.node.get_closest_marker("gpu"):
        request.getfixturevalue("cuda_lib")
