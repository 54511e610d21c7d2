"""The C ABI library without a GPU: it loads, exports every function the
public header declares, and its host-side argument checks reject bad input
before any CUDA call (no compute runs here)."""
import ctypes
import re
import subprocess
from pathlib import Path

import pytest

from thesiscode_b200 import _native as N

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module", autouse=True)
def _built(native_built):
    return native_built


def header_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(tc_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_header_declares_functions():
    assert len(header_functions()) >= 25


def test_library_exports_every_declared_symbol():
    exported = subprocess.run(["nm", "-D", "--defined-only", str(N.LIB_PATH)], capture_output=True,
                              text=True, check=True).stdout
    syms = set(re.findall(r"\bT (tc_[a-z0-9_]+)", exported))
    missing = [f for f in header_functions() if f not in syms]
    assert not missing, missing


def test_python_binding_covers_header():
    missing = [f for f in header_functions() if f not in N.SIGNATURES]
    assert not missing, missing


def test_library_is_built_for_sm_100a_only():
    out = subprocess.run(["cuobjdump", "--list-elf", str(N.LIB_PATH)], capture_output=True,
                         text=True).stdout
    assert "sm_100a" in out
    assert not re.search(r"sm_(?!100a)\d+", out)


def test_version_and_error_strings():
    assert b"sm_100a" in N.lib().tc_version()
    assert isinstance(N.lib().tc_last_error(), bytes)


def test_argument_errors_without_gpu():
    L = N.lib()
    # null output pointer / bad precision never reach CUDA
    assert L.tc_create(0, 0, None) == N.TC_ERR_ARG
    h = ctypes.c_void_p()
    assert L.tc_create(0, 7, ctypes.byref(h)) == N.TC_ERR_ARG
    assert L.tc_set_omega(None, 1.0) == N.TC_ERR_ARG
    v = ctypes.c_double()
    assert L.tc_probe_peak(0, 99, 10, ctypes.byref(v)) in (N.TC_ERR_ARG, N.TC_ERR_CUDA)
    assert L.tc_destroy(None) == N.TC_OK


def test_load_balance_host_mirror():
    from thesiscode_b200.panel_velocity import load_balance

    s, e = load_balance(10, 3)
    assert list(s) == [0, 3, 6] and list(e) == [3, 6, 10]
    s, e = load_balance(2, 4)  # more ranks than rows: empty leading chunks
    assert list(e - s) == [0, 0, 0, 2]


def test_c_load_balance_equals_oracle_partition():
    """tc_load_balance (the C ABI a C/Fortran host shards with) against the oracle's restatement of
    LoadBalance (PanelVelocityParallel.f90:182-204) and the Python mirror, including more ranks
    than rows; bad arguments are refused without a GPU."""
    from oracle import oracle as O
    from thesiscode_b200.panel_velocity import load_balance

    for n in (0, 1, 2, 7, 40962, 81920, 1310720):
        for p in (1, 2, 3, 4, 8, 16):
            s = (ctypes.c_int * p)()
            e = (ctypes.c_int * p)()
            N.call("tc_load_balance", n, p, s, e)
            os_, oe = O.load_balance(n, p)
            ps, pe = load_balance(n, p)
            assert list(s) == list(os_) == list(ps) and list(e) == list(oe) == list(pe), (n, p)
    s = (ctypes.c_int * 1)()
    assert N.lib().tc_load_balance(5, 0, s, s) == N.TC_ERR_ARG
    assert N.lib().tc_load_balance(-1, 1, s, s) == N.TC_ERR_ARG
    c = ctypes.c_int(-1)
    rc = N.lib().tc_device_count(ctypes.byref(c))
    assert (rc == N.TC_OK and c.value >= 1) or (rc == N.TC_ERR_CUDA and c.value == 0)
