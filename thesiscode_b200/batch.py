"""Batched ensembles of independent particle sets (tc_batch_rk4).

Each instance is a Workload (configs.Workload); the instances are copied back
to back, advanced `nsteps` RK4 steps on the GPU in one persistent launch per
stage (one CUDA graph for all steps when `graph`), and copied back in place.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native as N
from .panel_velocity import Context


def batch_rk4(ctx: Context, workloads, dt: float, nsteps: int, graph: bool = True,
              autotune: bool = True) -> np.ndarray:
    """Advance every workload by nsteps steps; returns totalKE with shape (nsteps, count)."""
    count = len(workloads)
    nA = np.array([w.nA for w in workloads], np.int32)
    nV = np.array([w.nV for w in workloads], np.int32)
    xA = np.ascontiguousarray(np.concatenate([w.xA for w in workloads]))
    zA = np.ascontiguousarray(np.concatenate([w.zetaA for w in workloads]))
    aA = np.ascontiguousarray(np.concatenate([w.areaA for w in workloads]))
    xV = np.ascontiguousarray(np.concatenate([w.xV for w in workloads]))
    tke = np.zeros(max(1, nsteps * count))
    flags = (N.TC_BATCH_GRAPH if graph else 0) | (N.TC_BATCH_AUTOTUNE if autotune else 0)
    N.call("tc_batch_rk4", ctx.handle, count, N.iptr(nA), N.iptr(nV), N.dptr(xA), N.dptr(zA), N.dptr(aA),
           N.dptr(xV), float(dt), int(nsteps), N.dptr(tke), flags)
    a = v = 0
    for w in workloads:
        w.xA[:] = xA[a:a + w.nA]
        w.zetaA[:] = zA[a:a + w.nA]
        w.xV[:] = xV[v:v + w.nV]
        a += w.nA
        v += w.nV
    return tke[:nsteps * count].reshape(nsteps, count)


def batch_info(ctx: Context) -> dict:
    v, c, n = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    N.call("tc_batch_info", ctx.handle, ctypes.byref(v), ctypes.byref(c), ctypes.byref(n))
    return {"variant": v.value, "chunk_len": c.value, "work_items": n.value}
