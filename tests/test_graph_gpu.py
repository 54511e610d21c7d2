"""tc_rk4_advance with its steps replayed from a CUDA graph (small problems) gives bitwise the
launch-by-launch results, counts the same kernels, replays the cached graph on the next call and
recaptures when the step changes."""
import ctypes

import numpy as np
import pytest

from thesiscode_b200 import _native as N
from thesiscode_b200 import configs
from thesiscode_b200.panel_velocity import Context

pytestmark = pytest.mark.gpu


def advance(w, precision, mode, dt, nsteps, calls=1):
    ctx = Context(0, precision)
    ctx.set_omega(w.omega)
    ctx.set_deltas(*w.deltas)
    N.call("tc_set_rk4_graphs", ctx.handle, mode)
    N.call("tc_rk4_load", ctx.handle, N.dptr(w.xA), N.dptr(w.zetaA), N.dptr(w.areaA), w.nA, N.dptr(w.xV),
           w.nV, N.dptr(w.xQ), w.nQ, 0)
    kes = []
    N.call("tc_stats", ctx.handle, 1, None, None, None, None)
    for _ in range(calls):
        tke = np.zeros(nsteps)
        N.call("tc_rk4_advance", ctx.handle, dt, nsteps, N.dptr(tke))
        kes.append(tke)
    launches, pairs = ctypes.c_longlong(), ctypes.c_longlong()
    N.call("tc_stats", ctx.handle, 0, ctypes.byref(launches), None, ctypes.byref(pairs), None)
    out = dict(xA=np.zeros((w.nA, 3)), zA=np.zeros(w.nA), xV=np.zeros((w.nV, 3)), xQ=np.zeros((w.nQ, 3)))
    N.call("tc_rk4_store", ctx.handle, N.dptr(out["xA"]), N.dptr(out["zA"]), N.dptr(out["xV"]),
           N.dptr(out["xQ"]), None, 0)
    ctx.close()
    out["tke"] = np.concatenate(kes)
    out["launches"], out["pairs"] = launches.value, pairs.value
    return out


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_graph_replay_is_bitwise_the_launch_path(gpu, precision):
    w = configs.rh4(level=3, parity=True, dt=0.01)
    ref = advance(w, precision, 0, w.dt, 5, calls=2)
    got = advance(w, precision, 2, w.dt, 5, calls=2)  # the second call replays the cached graph
    for k in ("xA", "zA", "xV", "xQ", "tke"):
        assert np.array_equal(got[k], ref[k]), k
    assert got["launches"] == ref["launches"] and got["pairs"] == ref["pairs"]


def test_graph_recaptures_when_the_step_changes(gpu):
    w = configs.rh4(level=3, parity=True, dt=0.01)
    ctx = Context(0, "fp64")
    ctx.set_omega(w.omega)
    ctx.set_deltas(*w.deltas)
    N.call("tc_set_rk4_graphs", ctx.handle, 2)
    N.call("tc_rk4_load", ctx.handle, N.dptr(w.xA), N.dptr(w.zetaA), N.dptr(w.areaA), w.nA, N.dptr(w.xV),
           w.nV, N.dptr(w.xQ), w.nQ, 0)
    N.call("tc_rk4_advance", ctx.handle, 0.01, 4, None)
    N.call("tc_rk4_advance", ctx.handle, 0.005, 4, None)
    xA = np.zeros((w.nA, 3))
    N.call("tc_rk4_store", ctx.handle, N.dptr(xA), None, None, None, None, 0)
    ctx.close()
    ctx = Context(0, "fp64")
    ctx.set_omega(w.omega)
    ctx.set_deltas(*w.deltas)
    N.call("tc_set_rk4_graphs", ctx.handle, 0)
    N.call("tc_rk4_load", ctx.handle, N.dptr(w.xA), N.dptr(w.zetaA), N.dptr(w.areaA), w.nA, N.dptr(w.xV),
           w.nV, N.dptr(w.xQ), w.nQ, 0)
    N.call("tc_rk4_advance", ctx.handle, 0.01, 4, None)
    N.call("tc_rk4_advance", ctx.handle, 0.005, 4, None)
    xB = np.zeros((w.nA, 3))
    N.call("tc_rk4_store", ctx.handle, N.dptr(xB), None, None, None, None, 0)
    ctx.close()
    assert np.array_equal(xA, xB)
    with pytest.raises(N.TcError):
        N.call("tc_set_rk4_graphs", None, 1)
