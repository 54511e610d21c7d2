import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def native_built():
    """Build the library and the oracle once per session (seconds when up to date)."""
    from thesiscode_b200 import build as b
    from oracle import oracle

    b.build()
    oracle.build()
    return True


@pytest.fixture(scope="session")
def gpu(native_built):
    """Fails (never skips) when the GPU tests run without a usable CUDA device."""
    import ctypes

    from thesiscode_b200 import _native as N

    v = ctypes.c_double()
    rc = N.lib().tc_probe_peak(0, N.TC_PROBE_FFMA, 16, ctypes.byref(v))
    if rc != 0:
        pytest.fail("GPU tests need a CUDA device: " + N.lib().tc_last_error().decode())
    return True
