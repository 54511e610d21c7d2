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
    """Build the library (and, with TC_LIBRARY=checked, its index-checked build) and the
    oracle once per session (seconds when up to date)."""
    from thesiscode_b200 import _native as N
    from thesiscode_b200 import build as b
    from oracle import oracle

    b.build()
    if N.CHECKED:
        b.build(checked=True)
    oracle.build()
    return True


@pytest.fixture(autouse=True)
def _index_checks_clean(request):
    """With the index-checked library loaded (TC_LIBRARY=checked), a GPU test fails when any
    kernel it launched indexed outside an array (the device's record is read and cleared)."""
    yield
    if request.node.get_closest_marker("gpu") is None:
        return
    from thesiscode_b200 import _native as N

    if not N.CHECKED or N._lib is None:
        return
    rec = N.bounds_status(0, reset=True)
    assert rec["count"] == 0, f"index check fired: {rec}"


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
