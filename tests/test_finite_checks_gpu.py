"""NaN/Inf handling of the host-array entry points. The inputs are scanned on the host while the GPU
already works on their device copies and the results are copied back only after the scan passed, so
a refused call returns TC_ERR_NONFINITE naming the array and the first bad index and leaves every
caller array as it was; results are scanned on the device and a non-finite one is reported with its
first index after the copy back (the reference returns such values silently); the context stays
usable after either."""
import ctypes

import numpy as np
import pytest

from thesiscode_b200 import _native as N
from thesiscode_b200 import configs
from thesiscode_b200.panel_velocity import Context

pytestmark = pytest.mark.gpu


def make_ctx(w, precision):
    ctx = Context(0, precision)
    ctx.set_omega(w.omega)
    ctx.set_deltas(*w.deltas)
    return ctx


def rk4_arrays(w):
    return w.xA.copy(), w.zetaA.copy(), w.xV.copy(), w.xQ.copy()


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_rk4_step_refuses_nan_input_and_leaves_arrays(gpu, precision):
    w = configs.rh4(level=2, parity=True)
    ctx = make_ctx(w, precision)
    xA, zA, xV, xQ = rk4_arrays(w)
    zA[7] = np.nan
    xV[3, 1] = np.inf
    before = [a.copy() for a in (xA, zA, xV, xQ)]
    with pytest.raises(N.TcError) as e:
        ctx.rk4_step(xA, zA, w.areaA, xV, xQ, w.dt, 2)
    assert e.value.status == N.TC_ERR_NONFINITE
    assert "zetaA at index 7" in str(e.value)
    for a, b in zip((xA, zA, xV, xQ), before):
        assert np.array_equal(a, b, equal_nan=True)
    # the state loaded from the refused inputs is dropped
    z = np.zeros(w.nA)
    assert N.lib().tc_rk4_store(ctx.handle, None, N.dptr(z), None, None, None, 0) == N.TC_ERR_STATE
    # and the next call gives what a fresh context gives
    got = rk4_arrays(w)
    ctx.rk4_step(got[0], got[1], w.areaA, got[2], got[3], w.dt, 2)
    ctx.close()
    ref = rk4_arrays(w)
    fresh = make_ctx(w, precision)
    fresh.rk4_step(ref[0], ref[1], w.areaA, ref[2], ref[3], w.dt, 2)
    fresh.close()
    for a, b in zip(got, ref):
        assert np.array_equal(a, b)


def test_rk4_step_names_the_first_bad_input(gpu):
    w = configs.rh4(level=2, parity=True)
    ctx = make_ctx(w, "fp64")
    xA, zA, xV, xQ = rk4_arrays(w)
    xV[5, 2] = np.nan
    with pytest.raises(N.TcError) as e:
        ctx.rk4_step(xA, zA, w.areaA, xV, xQ, w.dt, 1)
    assert e.value.status == N.TC_ERR_NONFINITE
    assert "xV at index 17" in str(e.value)
    ctx.close()


def test_velocity_refuses_nan_targets_and_leaves_outputs(gpu):
    w = configs.rh4(level=2, parity=True)
    ctx = make_ctx(w, "fp64")
    X = w.xV.copy()
    X[4, 0] = np.nan
    dX = np.full((w.nV, 3), 7.0)
    rc = N.lib().tc_bs_velocity(ctx.handle, N.TC_VERTEX, N.dptr(X), w.nV, N.dptr(w.xA), N.dptr(w.zetaA),
                                N.dptr(w.areaA), w.nA, 0, w.nV, N.dptr(dX), None)
    assert rc == N.TC_ERR_NONFINITE
    assert b"X at index 12" in N.lib().tc_last_error()
    assert np.all(dX == 7.0)
    dX, _ = ctx.velocity(N.TC_VERTEX, w.xV, w.xA, w.zetaA, w.areaA)
    assert np.all(np.isfinite(dX))
    ctx.close()


def first_bad(a):
    return int(np.flatnonzero(~np.isfinite(a.ravel()))[0])


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_non_finite_result_is_reported_with_its_index(gpu, precision):
    # finite inputs whose product zeta*A overflows: every other target row sees an infinite weight
    w = configs.rh4(level=2, parity=True)
    ctx = make_ctx(w, precision)
    vort, area = w.zetaA.copy(), w.areaA.copy()
    vort[3], area[3] = 1e300, 1e300
    dX, dV = np.zeros((w.nA, 3)), np.zeros(w.nA)
    rc = N.lib().tc_bs_velocity(ctx.handle, N.TC_ACTIVE, None, w.nA, N.dptr(w.xA), N.dptr(vort),
                                N.dptr(area), w.nA, 0, w.nA, N.dptr(dX), N.dptr(dV))
    assert rc == N.TC_ERR_NONFINITE
    # the results were copied back; the message names the first non-finite one
    assert f"dX (result) at index {first_bad(dX)}".encode() in N.lib().tc_last_error()
    dX, _ = ctx.velocity(N.TC_ACTIVE, None, w.xA, w.zetaA, w.areaA)
    assert np.all(np.isfinite(dX))
    ctx.close()


def test_rk4_step_reports_a_non_finite_result(gpu):
    w = configs.rh4(level=2, parity=True)
    ctx = make_ctx(w, "fp64")
    xA, zA, xV, xQ = rk4_arrays(w)
    area = w.areaA.copy()
    zA[3], area[3] = 1e300, 1e300
    with pytest.raises(N.TcError) as e:
        ctx.rk4_step(xA, zA, area, xV, xQ, w.dt, 1)
    assert e.value.status == N.TC_ERR_NONFINITE
    assert f"xA (result) at index {first_bad(xA)}" in str(e.value)
    ctx.close()


def test_soa_velocity_refuses_nan_input(gpu):
    w = configs.rh4(level=2, parity=True)
    ctx = make_ctx(w, "fp64")
    x, y, z = (np.ascontiguousarray(w.xA[:, c]) for c in range(3))
    y = y.copy()
    y[9] = np.nan
    dx, dy, dz, dv = np.full(w.nA, 5.0), np.zeros(w.nA), np.zeros(w.nA), np.full(w.nA, 5.0)
    rc = N.lib().tc_bs_velocity_soa(ctx.handle, N.dptr(x), N.dptr(y), N.dptr(z), N.dptr(w.zetaA),
                                    N.dptr(w.areaA), w.nA, 0, w.nA, N.dptr(dx), N.dptr(dy), N.dptr(dz),
                                    N.dptr(dv))
    assert rc == N.TC_ERR_NONFINITE
    assert b"y at index 9" in N.lib().tc_last_error()
    assert np.all(dx == 5.0) and np.all(dv == 5.0)
    ctx.close()


def test_strat_step_refuses_nan_vorticity_and_leaves_arrays(gpu):
    w = configs.stratosphere(level=2)
    ctx = make_ctx(w, "fp64")
    xA, xV, xQ = w.xA.copy(), w.xV.copy(), w.xQ.copy()
    absA = w.meta["absVortA"].copy()
    absA[11] = np.nan
    before = [a.copy() for a in (xA, xV, xQ)]
    with pytest.raises(N.TcError) as e:
        ctx.strat_rk4_step(xA, absA, w.areaA, xV, xQ, 0.0, w.dt, 1, absVortV=w.meta["absVortV"])
    assert e.value.status == N.TC_ERR_NONFINITE
    assert "absVortA at index 11" in str(e.value)
    for a, b in zip((xA, xV, xQ), before):
        assert np.array_equal(a, b)
    relA, relV, tke, _ = ctx.strat_rk4_step(xA, w.meta["absVortA"], w.areaA, xV, xQ, 0.0, w.dt, 1,
                                            absVortV=w.meta["absVortV"])
    assert np.all(np.isfinite(relA)) and np.all(np.isfinite(relV)) and np.all(np.isfinite(tke))
    ctx.close()
