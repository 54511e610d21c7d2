"""Checkpoint files of the device-resident RK4 state (tc_rk4_save / tc_rk4_restore).

The library writes and reads them (csrc/checkpoint.cu). `read` loads one into
numpy arrays for post-processing, on any machine: the file is validated by
the library's own reader (tc_rk4_checkpoint_info, which needs no GPU) and
then parsed here. Layout, little-endian:

    char[8] "TCB2RK4\\0"; u32 version (1); u32 flags (bit 0: forced run);
    i32 nA, nV, nQ, precision; i64 steps since load, forced step count;
    f64 Omega, delta[3], t0, forced step length;
    f64 xA[3nA], zetaA[nA], areaA[nA], xV[3nV], xQ[3nQ];
    forced runs also f64 absVortA[nA], absVortV[nV];
    u64 FNV-1a hash of every byte before it.
"""
from __future__ import annotations

import ctypes
import struct

import numpy as np

from . import _native as N

MAGIC = b"TCB2RK4\0"
VERSION = 1
HEADER = struct.Struct("<8sIIiiiiqq6d")  # 96 bytes


def info(path) -> dict:
    """Sizes, forced flag and step count of a valid checkpoint (TcError for a bad one)."""
    nA, nV, nQ, forced = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    steps = ctypes.c_longlong()
    N.call("tc_rk4_checkpoint_info", str(path).encode(), ctypes.byref(nA), ctypes.byref(nV),
           ctypes.byref(nQ), ctypes.byref(forced), ctypes.byref(steps))
    return {"nA": nA.value, "nV": nV.value, "nQ": nQ.value, "forced": bool(forced.value),
            "steps": steps.value}


def read(path) -> dict:
    """The arrays and parameters of a checkpoint (TcError for a bad file)."""
    info(path)
    raw = open(path, "rb").read()
    (_, _, flags, nA, nV, nQ, precision, steps, fstep, omega, d0, d1, d2, t0,
     dt) = HEADER.unpack_from(raw)
    forced = bool(flags & 1)
    counts = [3 * nA, nA, nA, 3 * nV, 3 * nQ] + ([nA, nV] if forced else [])
    v = np.frombuffer(raw, dtype="<f8", count=sum(counts), offset=HEADER.size)
    parts = np.split(v, np.cumsum(counts)[:-1])
    out = {"xA": parts[0].reshape(nA, 3), "zetaA": parts[1], "areaA": parts[2],
           "xV": parts[3].reshape(nV, 3), "xQ": parts[4].reshape(nQ, 3), "omega": omega,
           "deltas": (d0, d1, d2), "steps": steps, "precision": precision, "forced": forced}
    if forced:
        out.update(absVortA=parts[5], absVortV=parts[6], t0=t0, forced_step=fstep, dt=dt)
    return out
