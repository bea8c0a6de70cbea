import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "voss-prime-gaps_v1_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the native kernels")
    config.addinivalue_line("markers", "slow: long-running")


def _has_gpu() -> bool:
    try:
        import voss
        return voss.device_count() > 0
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu_ctx():
    """One context for the GPU tests, able to sieve up to 10^13."""
    import voss
    if not _has_gpu():
        pytest.fail("a -m gpu test ran without a CUDA device or without libvoss.so")
    ctx = voss.Context(10**13 + 10**9)
    yield ctx
    ctx.close()


@pytest.fixture(scope="session")
def gpu_ctx_big():
    """A context whose base-prime table reaches 10^9 (intervals up to 10^18)."""
    import voss
    if not _has_gpu():
        pytest.fail("a -m gpu test ran without a CUDA device or without libvoss.so")
    ctx = voss.Context(10**18 + 2 * 10**9)
    yield ctx
    ctx.close()
