import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the product library's numeric phase")


def _gpu_available() -> bool:
    try:
        from rustyfem_b200 import ffi

        return ffi.device_count() > 0
    except Exception:
        return False


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Builds the libraries once per session (a no-op when they are up to date)."""
    from oracle import refcpu
    from rustyfem_b200 import _build

    _build.build_mesh()
    _build.build_gpu()
    refcpu.build()
    yield


@pytest.fixture(scope="session")
def gpu():
    from rustyfem_b200 import ffi

    if ffi.device_count() < 1:
        pytest.fail("a gpu-marked test ran without a CUDA device")
    return True
