import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests through the C ABI")


def _has_gpu():
    try:
        from spaqr_public_b200 import _abi
        import ctypes
        n = ctypes.c_int(0)
        return _abi.lib().spq_device_count(ctypes.byref(n)) == 0 and n.value > 0
    except Exception:
        return False


@pytest.fixture(scope="session", autouse=True)
def built_libraries():
    """Builds the CUDA library and the CPU oracle once if they are missing."""
    from spaqr_public_b200 import build
    lib = os.path.join(ROOT, "spaqr_public_b200", "_build", "libspaqr_b200.so")
    orc = os.path.join(ROOT, "oracle", "_build", "liboracle.so")
    if not (os.path.exists(lib) and os.path.exists(orc)):
        build.build()
    yield


@pytest.fixture(scope="session")
def gpu():
    if not _has_gpu():
        pytest.fail("no CUDA device visible: GPU tests need a B200")
    return True
