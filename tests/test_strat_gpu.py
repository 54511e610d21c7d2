"""Forced (stratosphere) RK4 step on the GPU (tc_strat_rk4_step) against the
FP64 oracle's restatement of StratosphereRK4 (PanelVelocityParallel.f90:661-919).

Error metric: max |x_gpu - x_ref| / max |x_new - x_old| for positions and
max |zeta_gpu - zeta_ref| / max |zeta_ref| for the relative vorticity.
Tolerances: FP64 1e-12; FP32-compensated 5e-7 (level 3, the coarse-grid bound of the BVE step).
"""
import numpy as np
import pytest

from oracle import oracle as O
from thesiscode_b200 import _native as N
from thesiscode_b200 import configs, grid
from thesiscode_b200.panel_velocity import Context, PanelVelocity

pytestmark = pytest.mark.gpu


def oracle_steps(w, t0, nsteps):
    xV, xA, xQ = w.xV.copy(), w.xA.copy(), w.xQ.copy()
    absA, absV = w.meta["absVortA"], w.meta["absVortV"]
    tke = []
    for k in range(nsteps):
        xV, xA, relA, xQ, ke_tot, ke, relV = O.strat_rk4(xV, xA, absA, w.areaA, xQ, t0 + k * w.dt, w.dt,
                                                         w.omega, w.deltas, absVortV=absV, nthreads=8)
        tke.append(ke_tot)
    return xV, xA, relA, xQ, np.array(tke), relV


def gpu_steps(w, t0, nsteps, precision):
    ctx = Context(0, precision)
    ctx.set_omega(w.omega)
    ctx.set_deltas(*w.deltas)
    xA, xV, xQ = w.xA.copy(), w.xV.copy(), w.xQ.copy()
    relA, relV, tke, ke = ctx.strat_rk4_step(xA, w.meta["absVortA"], w.areaA, xV, xQ, t0, w.dt, nsteps,
                                             absVortV=w.meta["absVortV"])
    ctx.close()
    return xV, xA, relA, xQ, tke, relV


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32c", 5e-7)])
@pytest.mark.parametrize("t0", [5.0, 2.0])  # full forcing; ramp-up (A(t) varies within the step)
def test_strat_rk4_matches_oracle(gpu, precision, tol, t0):
    w = configs.stratosphere(level=3, dt=0.01)
    ref = oracle_steps(w, t0, 2)
    got = gpu_steps(w, t0, 2, precision)
    for r, g, x0 in ((ref[0], got[0], w.xV), (ref[1], got[1], w.xA), (ref[3], got[3], w.xQ)):
        assert np.abs(g - r).max() <= tol * np.abs(r - x0).max()
    for r, g in ((ref[2], got[2]), (ref[5], got[5])):
        assert np.abs(g - r).max() <= tol * np.abs(r).max()
    assert np.abs(got[4] - ref[4]).max() <= 2 * tol * np.abs(ref[4]).max()


def test_strat_without_forcing_equals_bve_step(gpu):
    w = configs.stratosphere(level=3, dt=0.01)
    absA = w.meta["absVortA"]
    ctx = Context(0, "fp64")
    ctx.set_omega(w.omega)
    ctx.set_deltas(*w.deltas)
    xA, xV, xQ = w.xA.copy(), w.xV.copy(), w.xQ.copy()
    relA, _, tke_s, _ = ctx.strat_rk4_step(xA, absA, w.areaA, xV, xQ, 20.0, w.dt, 3)
    xB, xVB, xQB = w.xA.copy(), w.xV.copy(), w.xQ.copy()
    zB = absA - 2.0 * w.omega * w.xA[:, 2]
    tke_b, _ = ctx.rk4_step(xB, zB, w.areaA, xVB, xQB, w.dt, 3)
    disp = np.abs(xB - w.xA).max()
    assert np.abs(xA - xB).max() <= 1e-12 * disp
    assert np.abs(xV - xVB).max() <= 1e-12 * disp
    assert np.abs(relA - zB).max() <= 1e-12 * np.abs(zB).max()
    assert np.abs(tke_s - tke_b).max() <= 1e-12 * tke_b.max()
    ctx.close()


def test_strat_zero_steps_returns_rel_vort_at_t(gpu):
    w = configs.stratosphere(level=2, dt=0.01)
    ctx = Context(0, "fp64")
    xA, xV, xQ = w.xA.copy(), w.xV.copy(), w.xQ.copy()
    relA, relV, tke, _ = ctx.strat_rk4_step(xA, w.meta["absVortA"], w.areaA, xV, xQ, 5.0, w.dt, 0,
                                            absVortV=w.meta["absVortV"])
    expect = w.meta["absVortA"] - 2.0 * w.omega * w.xA[:, 2] - O.juckes_forcing(w.xA, 5.0)
    assert np.abs(relA - expect).max() <= 1e-13 * np.abs(expect).max()
    expectV = w.meta["absVortV"] - 2.0 * w.omega * w.xV[:, 2] - O.juckes_forcing(w.xV, 5.0)
    assert np.abs(relV - expectV).max() <= 1e-13 * np.abs(expectV).max()
    assert np.array_equal(xA, w.xA)
    with pytest.raises(N.TcError):
        ctx.strat_rk4_step(xA, w.meta["absVortA"], w.areaA, xV, xQ, float("nan"), w.dt, 1)
    ctx.close()


def test_module_mirror_stratosphere_rk4(gpu):
    """PanelVelocity.StratosphereRK4 on the reference's Particles/Panels types."""
    parts, pans = grid.new_icos_grid(3)
    w = configs.stratosphere(level=3, dt=0.01)
    maps = grid.gather_maps(pans)
    pans.absVort[maps.active] = w.meta["absVortA"]
    pans.relVort[maps.active] = w.zetaA
    parts.absVort[:] = w.meta["absVortV"]
    pv = PanelVelocity(0, "fp64")
    pv.StratosphereRK4(parts, pans, 5.0, w.dt)
    ref = oracle_steps(w, 5.0, 1)
    assert np.abs(parts.x - ref[0]).max() <= 1e-12 * np.abs(ref[0] - w.xV).max()
    assert np.abs(pans.relVort[maps.active] - ref[2]).max() <= 1e-12 * np.abs(ref[2]).max()
    assert np.abs(parts.relVort - ref[5]).max() <= 1e-12 * np.abs(ref[5]).max()
    assert pv.totalKE > 0
