import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libscpgpu.so")
    config.addinivalue_line("markers", "slow: long CPU reference runs")


def gpu_available() -> bool:
    try:
        import ctypes
        cudart = None
        for name in ("libcuda.so.1", "libcuda.so"):
            try:
                cudart = ctypes.CDLL(name)
                break
            except OSError:
                continue
        if cudart is None:
            return False
        n = ctypes.c_int(0)
        if cudart.cuInit(0) != 0:
            return False
        return cudart.cuDeviceGetCount(ctypes.byref(n)) == 0 and n.value > 0
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    if not gpu_available():
        pytest.fail("GPU test selected but no CUDA device is visible")
    from scp_b200 import native
    native.lib()
    return True


@pytest.fixture(scope="session")
def reference():
    """The reference's own CPU binary (oracle/_ref, built from the reference
    tree by `make -C oracle ref`); tests that run it skip without it."""
    import oracle
    if not oracle.reference_available():
        pytest.skip("reference binary not built (make -C oracle ref needs the reference tree)")
    return True
