import os
import sys

import pytest

# One stream-ordered pool for torch and the kernels' scratch (set before
# torch first touches CUDA).
os.environ.setdefault("PYTORCH_CUDA_ALLOC_CONF", "backend:cudaMallocAsync")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


@pytest.fixture(autouse=True)
def _device_errors_checked(request):
    """After every test that used an executor `ex`, synchronise it so a
    device-side failure (bounded look-back expiry, bounds check) is reported
    by the test that caused it."""
    yield
    ex = getattr(request.node, "funcargs", {}).get("ex")
    if ex is not None and hasattr(ex, "sync"):
        ex.sync()


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle
    return oracle
