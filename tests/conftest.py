import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA path through the C ABI")


def _ensure_built():
    """Builds the oracle checkers and libmgm.so if they are missing or stale."""
    orc = os.path.join(ROOT, "oracle")
    if not (os.path.exists(os.path.join(orc, "liboracle.so")) and os.path.exists(os.path.join(orc, "liboracle_crpow.so"))):
        subprocess.run(["make", "-C", orc, "liboracle.so", "liboracle_crpow.so"], check=True, capture_output=True)
    from multigrid_meshless_b200 import build
    build.build()


_ensure_built()


def gpu_available() -> bool:
    try:
        import ctypes
        cudart = None
        for name in ("libcudart.so", "libcudart.so.12"):
            try:
                cudart = ctypes.CDLL(name)
                break
            except OSError:
                continue
        if cudart is None:
            import torch
            return torch.cuda.is_available()
        n = ctypes.c_int(0)
        return cudart.cudaGetDeviceCount(ctypes.byref(n)) == 0 and n.value > 0
    except Exception:
        return False


@pytest.fixture(scope="session")
def require_gpu():
    if not gpu_available():
        pytest.fail("this test needs a CUDA device (run with -m 'not gpu' on machines without one)")
