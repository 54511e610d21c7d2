"""ctypes binding of libthesiscode_b200.so (the C ABI in include/thesiscode_b200.h).

The library is the product: there is no Python or CPU fallback. Loading
fails with an ImportError naming the missing file when it has not been
built (``python -m thesiscode_b200.build``); calls that need a GPU return
the library's CUDA status, which is raised as ``TcError``.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_int, c_void_p
from pathlib import Path

LIB_DIR = Path(__file__).resolve().parent / "_lib"
# TC_LIBRARY=checked loads the build whose hot-path kernels check every
# global-memory index (tc_bounds_*); anything else loads the release build.
CHECKED = os.environ.get("TC_LIBRARY", "") == "checked"
LIB_PATH = LIB_DIR / ("libthesiscode_b200_checked.so" if CHECKED else "libthesiscode_b200.so")

# status codes
TC_OK = 0
TC_ERR_ARG = -1
TC_ERR_CUDA = -2
TC_ERR_NONFINITE = -3
TC_ERR_TIMEOUT = -4
TC_ERR_STATE = -5
TC_ERR_NOMEM = -6
# precision
TC_FP64 = 0
TC_FP32C = 1
# FP32C target visiting order
TC_ORDER_GIVEN = 0
TC_ORDER_HILBERT = 1
# target classes
TC_ACTIVE = 0
TC_VERTEX = 1
TC_PASSIVE = 2
# probes
(TC_PROBE_FFMA, TC_PROBE_FFMA2, TC_PROBE_DFMA, TC_PROBE_RCP32, TC_PROBE_RCP64, TC_PROBE_DDIV,
 TC_PROBE_F2F, TC_PROBE_FAR_PAIRS) = range(8)
# batched ensembles
TC_BATCH_GRAPH = 1
TC_BATCH_AUTOTUNE = 2
# adjoint functionals
TC_J_ENSTROPHY = 0
TC_J_PROBE = 1
# RK4 device buffers
TC_BUF_SOURCES, TC_BUF_XA, TC_BUF_ZETA, TC_BUF_XV, TC_BUF_XQ, TC_BUF_KE = range(6)
# index-check sites of the checked build (TC_BC_*), by id
BC_SITES = {
    1: "pair target positions", 2: "pair visiting order", 3: "pair packed sources",
    4: "pair partial-sum stores", 5: "batch segment table", 6: "packing inputs",
    7: "packing stores", 8: "velocity epilogue visiting order",
    9: "velocity epilogue target positions", 10: "velocity epilogue partial sums",
    11: "velocity epilogue stores", 12: "stage epilogue visiting orders",
    13: "stage epilogue state arrays", 14: "stage epilogue partial sums",
    15: "stage epilogue chunk counts", 16: "stage epilogue active-only arrays",
    17: "stage epilogue KE block sums", 18: "adjoint row-pass inputs",
    19: "adjoint row-pass partial stores", 20: "adjoint combination partial reads",
    21: "visiting-order key inputs", 22: "visiting-order key stores",
    23: "batch KE sums' reads",
}

_STATUS = {
    TC_ERR_ARG: "bad argument",
    TC_ERR_CUDA: "CUDA error",
    TC_ERR_NONFINITE: "non-finite value",
    TC_ERR_TIMEOUT: "device wait timed out",
    TC_ERR_STATE: "call out of sequence",
    TC_ERR_NOMEM: "out of memory",
}

dp = POINTER(c_double)
ip = POINTER(c_int)

# name -> (restype, argtypes); the argument lists mirror the header.
SIGNATURES: dict[str, tuple] = {
    "tc_version": (c_char_p, []),
    "tc_last_error": (c_char_p, []),
    "tc_probe_peak": (c_int, [c_int, c_int, c_int, dp]),
    "tc_create": (c_int, [c_int, c_int, POINTER(c_void_p)]),
    "tc_destroy": (c_int, [c_void_p]),
    "tc_set_stream": (c_int, [c_void_p, c_void_p]),
    "tc_synchronize": (c_int, [c_void_p]),
    "tc_set_precision": (c_int, [c_void_p, c_int]),
    "tc_get_precision": (c_int, [c_void_p, ip]),
    "tc_set_omega": (c_int, [c_void_p, c_double]),
    "tc_get_omega": (c_int, [c_void_p, dp]),
    "tc_set_smooth": (c_int, [c_void_p, c_double]),
    "tc_get_smooth": (c_int, [c_void_p, dp]),
    "tc_set_target_order": (c_int, [c_void_p, c_int]),
    "tc_set_adjoint_mode": (c_int, [c_void_p, c_int]),
    "tc_adjoint_phase_ms": (c_int, [c_void_p, dp]),
    "tc_set_deltas": (c_int, [c_void_p, c_double, c_double, c_double]),
    "tc_get_deltas": (c_int, [c_void_p, dp]),
    "tc_bs_velocity": (c_int, [c_void_p, c_int, dp, c_int, dp, dp, dp, c_int, c_int, c_int, dp, dp]),
    "tc_bs_velocity_device": (c_int, [c_void_p, c_int, c_void_p, c_int, c_void_p, c_void_p, c_void_p,
                                      c_int, c_int, c_int, c_void_p, c_void_p]),
    "tc_bs_velocity_device_noalloc": (c_int, [c_void_p, c_int, c_void_p, c_int, c_void_p, c_void_p,
                                              c_void_p, c_int, c_int, c_int, c_void_p, c_void_p]),
    "tc_bs_velocity_soa": (c_int, [c_void_p, dp, dp, dp, dp, dp, c_int, c_int, c_int, dp, dp, dp, dp]),
    "tc_bs_velocity_soa_device": (c_int, [c_void_p] + [c_void_p] * 5 + [c_int] * 3 + [c_void_p] * 4),
    "tc_rk4_soa_step": (c_int, [c_void_p, dp, dp, dp, dp, dp, c_int, c_double, c_int, dp, dp]),
    "tc_rk4_step": (c_int, [c_void_p, dp, dp, dp, c_int, dp, c_int, dp, c_int, c_double, c_int, dp, dp]),
    "tc_set_rk4_graphs": (c_int, [c_void_p, c_int]),
    "tc_rk4_vjp": (c_int, [c_void_p, dp, dp, dp, c_int, c_double, c_int, c_int, dp, dp, dp, dp, dp]),
    "tc_strat_rk4_step": (c_int, [c_void_p, dp, dp, dp, dp, c_int, dp, dp, dp, c_int, dp, c_int,
                                  c_double, c_double, c_int, dp, dp]),
    "tc_rk4_step_device": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_int,
                                   c_void_p, c_int, c_double, c_int, dp, c_void_p]),
    "tc_rk4_load": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_int, c_void_p,
                            c_int, c_int]),
    "tc_rk4_advance": (c_int, [c_void_p, c_double, c_int, dp]),
    "tc_rk4_store": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int]),
    "tc_load_balance": (c_int, [c_int, c_int, ip, ip]),
    "tc_device_count": (c_int, [ip]),
    "tc_reset_rk4": (c_int, [c_void_p]),
    "tc_rk4_pack_sources": (c_int, [c_void_p]),
    "tc_rk4_stage_range": (c_int, [c_void_p, c_int, c_double, c_int, c_int, c_int, c_int, c_int, c_int,
                                   c_void_p]),
    "tc_rk4_device_buffer": (c_int, [c_void_p, c_int, POINTER(c_void_p)]),
    "tc_batch_rk4": (c_int, [c_void_p, c_int, ip, ip, dp, dp, dp, dp, c_double, c_int, dp, c_int]),
    "tc_batch_info": (c_int, [c_void_p, ip, ip, ip]),
    "tc_rk4_adjoint": (c_int, [c_void_p, dp, dp, dp, c_int, c_double, c_int, c_int, c_int, c_int, dp, dp, dp]),
    "tc_rk4_copy_rows": (c_int, [c_void_p, c_int, c_int, c_int, c_void_p, c_int]),
    "tc_pair_variant_count": (c_int, [c_int, ip]),
    "tc_pair_variant_info": (c_int, [c_int, c_int, ip]),
    "tc_set_pair_variant": (c_int, [c_void_p, c_int, c_int]),
    "tc_get_pair_variant": (c_int, [c_void_p, c_int, ip]),
    "tc_stats_enable_timing": (c_int, [c_void_p, c_int]),
    "tc_stats": (c_int, [c_void_p, c_int, POINTER(ctypes.c_longlong), POINTER(ctypes.c_longlong),
                         POINTER(ctypes.c_longlong), dp]),
    "tc_icos_grid_sizes": (c_int, [c_int, ip, ip, ip, ip]),
    "tc_icos_grid": (c_int, [c_int, dp, dp, dp, dp, dp, ip, ip, ip, ip]),
    "tc_icos_grid_device": (c_int, [c_void_p, c_int] + [c_void_p] * 9),
    "tc_gather_maps": (c_int, [c_int, ip, ip, c_int, ip, c_int]),
    "tc_rk4_save": (c_int, [c_void_p, c_char_p]),
    "tc_rk4_restore": (c_int, [c_void_p, c_char_p]),
    "tc_rk4_steps_done": (c_int, [c_void_p, POINTER(ctypes.c_longlong)]),
    "tc_rk4_checkpoint_info": (c_int, [c_char_p, ip, ip, ip, ip, POINTER(ctypes.c_longlong)]),
    "tc_bounds_checked": (c_int, []),
    "tc_bounds_status": (c_int, [c_int, POINTER(ctypes.c_longlong), c_int]),
    "tc_bounds_cap": (c_int, [c_void_p, c_int, ctypes.c_longlong]),
}


class TcError(RuntimeError):
    """A negative status from the library, with tc_last_error()'s message."""

    def __init__(self, status: int, where: str, message: str):
        self.status = status
        super().__init__(f"{where}: {_STATUS.get(status, 'error')} ({status}): {message}")


_lib = None


def lib() -> ctypes.CDLL:
    """The loaded library (loads on first use; ImportError if it is not built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"{LIB_PATH} is missing: build the sm_100a library with "
                f"`python -m thesiscode_b200.build{' --checked' if CHECKED else ''}` "
                "(no CPU fallback exists)")
        handle = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def check(status: int, where: str) -> None:
    if status != TC_OK:
        msg = lib().tc_last_error().decode(errors="replace")
        raise TcError(status, where, msg)


def call(name: str, *args) -> None:
    """Call `name` and raise TcError on a negative status."""
    check(getattr(lib(), name)(*args), name)


def dptr(a) -> ctypes._Pointer:
    """double* of a C-contiguous float64 numpy array (or None)."""
    if a is None:
        return None
    return a.ctypes.data_as(dp)


def iptr(a) -> ctypes._Pointer:
    if a is None:
        return None
    return a.ctypes.data_as(ip)


def bounds_status(device: int = 0, reset: bool = False) -> dict:
    """The device's index-check record (checked build; zeros in the release
    build): violations, and site, index and extent of the first."""
    rec = (ctypes.c_longlong * 4)()
    call("tc_bounds_status", device, rec, 1 if reset else 0)
    return {"count": rec[0], "site": rec[1], "site_name": BC_SITES.get(rec[1], ""),
            "index": rec[2], "extent": rec[3]}
