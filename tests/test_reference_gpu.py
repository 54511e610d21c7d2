"""The library on the GPU against the reference's own code.

tests/golden/ref_*.npz hold what the reference's Fortran statements computed,
run through oracle/f90 (tests/golden/make_reference_fixtures.py): its grid and
initial conditions, BVERK4 and StratosphereRK4 on several MPI ranks, the
three RHS sums on partial index ranges, and the Voronoi BVEVelocity and BVERK4
(PanelVelocityParallel.f90:435-919,1287-1412; VoronoiVelocityParallel.f90:300-515).
Here the library computes the same steps and sums through the C ABI, and
through the drop-in host mirror of the reference's interface (BVERK4 on
Particles/Panels), and is compared with them.

Error metric: max |result - reference| / max |reference| of each velocity, and
of each RK4 displacement x_new - x_old (vorticity change for zeta). Tolerances:
FP64 1e-12; FP32C 5e-7, the stated bound at levels <= 3; kinetic energy twice
the velocity's (it is quadratic in u).
"""
from pathlib import Path

import numpy as np
import pytest

from thesiscode_b200 import _native as N
from thesiscode_b200 import grid
from thesiscode_b200.panel_velocity import Context, PanelVelocity
from thesiscode_b200.voronoi_velocity import BVEVelocity

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
OMEGA = 2 * np.pi
DELTAS = (0.0, 0.0, 0.05)
TOL = {"fp64": 1e-12, "fp32c": 5e-7}


def _load(name):
    return dict(np.load(GOLDEN / f"{name}.npz"))


def _state(f, prefix):
    n = len(prefix) + 1
    return {k[n:]: np.array(v) for k, v in f.items() if k.startswith(prefix + "_")}


def rel_err(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _ctx(prec):
    c = Context(0, prec)
    c.set_omega(OMEGA)
    c.set_deltas(*DELTAS)
    return c


@pytest.mark.parametrize("prec", ["fp64", "fp32c"])
@pytest.mark.parametrize("name", ["ref_bverk4_rh4_l2", "ref_bverk4_gauss_l2", "ref_bverk4_jet_l2",
                                  "ref_bverk4_rh4_l3"])
def test_rk4_step_equals_reference_bverk4(name, prec, gpu):
    f = _load(name)
    s0, s1 = _state(f, "initial"), _state(f, "final")
    ctx = _ctx(prec)
    xA, zA, xV, xQ = (s0[k].copy() for k in ("xA", "zetaA", "xV", "xQ"))
    tke, ke = ctx.rk4_step(xA, zA, s0["areaA"], xV, xQ, float(f["dt"]), int(f["steps"]))
    ctx.close()
    tol = TOL[prec]
    for k, new in (("xA", xA), ("xV", xV), ("xQ", xQ), ("zetaA", zA)):
        assert rel_err(new - s0[k], s1[k] - s0[k]) <= tol, k
    assert rel_err(tke, f["totalKE"]) <= 2 * tol
    assert rel_err(ke, f["kineticEnergy"]) <= 2 * tol


@pytest.mark.parametrize("prec", ["fp64", "fp32c"])
def test_host_mirror_bverk4_equals_reference(prec, gpu):
    """The drop-in: BVERK4(aParticles, aPanels, dt) on the library's own grid (equal bit for bit to
    the reference's) with the reference's initial vorticity, two steps, against the reference's
    BVERK4 on three ranks; includes the particles' relVort (:651) and the scatter back."""
    f = _load("ref_bverk4_rh4_l2")
    s0, s1 = _state(f, "initial"), _state(f, "final")
    parts, pans = grid.new_icos_grid(2)
    act = np.nonzero(~pans.hasChildren)[0]
    pas = np.nonzero(pans.hasChildren)[0]
    assert np.array_equal(pans.x[act], s0["xA"]) and np.array_equal(parts.x, s0["xV"])
    pans.relVort[act] = s0["zetaA"]
    pans.absVort[act] = s0["absVortA"]
    parts.relVort[:] = s0["relVortV"]
    parts.absVort[:] = s0["absVortV"]
    pv = PanelVelocity(0, prec)
    pv.SetOmega(OMEGA)
    pv.SetSmooth(0.05)
    tke = []
    for _ in range(int(f["steps"])):
        pv.BVERK4(parts, pans, float(f["dt"]))
        tke.append(pv.totalKE)
    tol = TOL[prec]
    assert rel_err(pans.x[act] - s0["xA"], s1["xA"] - s0["xA"]) <= tol
    assert rel_err(pans.x[pas] - s0["xQ"], s1["xQ"] - s0["xQ"]) <= tol
    assert rel_err(parts.x - s0["xV"], s1["xV"] - s0["xV"]) <= tol
    assert rel_err(pans.relVort[act] - s0["zetaA"], s1["zetaA"] - s0["zetaA"]) <= tol
    assert rel_err(parts.relVort, s1["relVortV"]) <= tol
    assert rel_err(np.array(tke), f["totalKE"]) <= 2 * tol


@pytest.mark.parametrize("prec", ["fp64", "fp32c"])
def test_stratosphere_step_equals_reference(prec, gpu):
    f = _load("ref_strat_l2")
    s0, s1 = _state(f, "initial"), _state(f, "final")
    ctx = _ctx(prec)
    xA, xV, xQ = s0["xA"].copy(), s0["xV"].copy(), s0["xQ"].copy()
    relA, relV, _, _ = ctx.strat_rk4_step(xA, s0["absVortA"], s0["areaA"], xV, xQ, float(f["t0"]),
                                          float(f["dt"]), int(f["steps"]), absVortV=s0["absVortV"])
    ctx.close()
    tol = TOL[prec]
    for k, new in (("xA", xA), ("xV", xV), ("xQ", xQ)):
        assert rel_err(new - s0[k], s1[k] - s0[k]) <= tol, k
    assert rel_err(relA, s1["zetaA"]) <= tol
    assert rel_err(relV, s1["relVortV"]) <= tol


@pytest.mark.parametrize("prec", ["fp64", "fp32c"])
def test_sums_equal_reference_rhs(prec, gpu):
    f = _load("ref_rhs_l2")
    xA, zA, aA = f["xA"], f["zetaA"], f["areaA"]
    ctx = _ctx(prec)
    tol = TOL[prec]
    a0, a1 = (int(v) for v in f["active_range"])
    dX, dV = ctx.velocity(N.TC_ACTIVE, None, xA, zA, aA, a0, a1)
    assert rel_err(dX, f["active_dX"]) <= tol
    assert rel_err(dV, f["active_dVort"]) <= tol
    assert np.all(dX[:a0] == 0) and np.all(dX[a1:] == 0)
    v0, v1 = (int(v) for v in f["vertex_range"])
    dX, _ = ctx.velocity(N.TC_VERTEX, f["xV"], xA, zA, aA, v0, v1)
    assert rel_err(dX, f["vertex_dX"]) <= tol
    dX, _ = ctx.velocity(N.TC_PASSIVE, f["xQ"], xA, zA, aA)
    assert rel_err(dX, f["passive_dX"]) <= tol
    r0, r1 = (int(v) for v in f["voronoi_range"])
    out = BVEVelocity(ctx, xA[:, 0], xA[:, 1], xA[:, 2], zA, aA, r0, r1, dy=f["voronoi_dy0"],
                      dz=f["voronoi_dz0"])
    for got, key in zip(out, ("voronoi_dx", "voronoi_dy", "voronoi_dz", "voronoi_dVort")):
        assert rel_err(got, f[key]) <= tol, key
    ctx.close()


@pytest.mark.parametrize("prec", ["fp64", "fp32c"])
def test_voronoi_rk4_equals_reference(prec, gpu):
    """BVERK4 of the Voronoi solver (VoronoiVelocityParallel.f90:300-483; its STRIPACK rebuild after
    the step is the caller's) on generators 1..N of arrays of N_Max > N slots, two steps."""
    from thesiscode_b200.voronoi_velocity import BVERK4, VorPanels

    f = _load("ref_voronoi_rk4_l2")
    s0, s1 = _state(f, "initial"), _state(f, "final")
    n = int(f["n"])
    vp = VorPanels(x=s0["x"].copy(), y=s0["y"].copy(), z=s0["z"].copy(), relVort=s0["relVort"].copy(),
                   absVort=s0["relVort"] + 2 * OMEGA * s0["z"], area=s0["area"].copy(), N=n)
    ctx = _ctx(prec)
    tke, _ = BVERK4(ctx, vp, float(f["dt"]), int(f["steps"]))
    ctx.close()
    tol = TOL[prec]
    for k in ("x", "y", "z", "relVort"):
        assert rel_err(getattr(vp, k)[:n] - s0[k][:n], s1[k] - s0[k][:n]) <= tol, k
    assert rel_err(tke, s1["totalKE"]) <= 2 * tol
