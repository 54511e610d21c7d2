"""Voronoi SoA path (BVEVelocity, VoronoiVelocityParallel.f90:487-515, and its BVERK4) on the GPU
against the oracle's golden fixture and the oracle RK4."""
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from thesiscode_b200 import configs
from thesiscode_b200.panel_velocity import Context
from thesiscode_b200.voronoi_velocity import BVERK4, BVEVelocity, VorPanels

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
TOL = {"fp64": 1e-12, "fp32c": 5e-7}  # levels 2-3: the coarse-grid FP32C bound


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("prec", ["fp64", "fp32c"])
def test_bvevelocity_golden_with_unused_slots(prec, gpu):
    g = np.load(GOLDEN / "voronoi_l2.npz")
    ctx = Context(0, prec)
    ctx.set_omega(float(g["omega"]))
    ctx.set_deltas(0.0, 0.0, 0.0)
    dx, dy, dz, dV = BVEVelocity(ctx, g["x"], g["y"], g["z"], g["vort"], g["area"], 0, int(g["n"]))
    ref = np.stack([g["dx"], g["dy"], g["dz"]], 1)
    assert rel(np.stack([dx, dy, dz], 1), ref) <= TOL[prec]
    assert rel(dV, g["dV"]) <= TOL[prec]
    ctx.close()


def test_bvevelocity_dy_dz_accumulate_like_reference(gpu):
    w = configs.rh4(level=2, parity=False)
    x, y, z = w.xA[:, 0], w.xA[:, 1], w.xA[:, 2]
    ctx = Context(0, "fp64")
    ctx.set_omega(w.omega)
    ctx.set_deltas(0.0, 0.0, 0.0)
    ones = np.ones(w.nA)
    got = BVEVelocity(ctx, x, y, z, w.zetaA, w.areaA, 5, 200, dy=ones, dz=2 * ones)
    ref = O.voronoi_velocity(x, y, z, w.zetaA, w.areaA, 5, 200, omega=w.omega, dy=ones, dz=2 * ones)
    for a, b in zip(got, ref):
        np.testing.assert_allclose(a, b, rtol=0, atol=1e-12 * np.abs(b).max())
    ctx.close()


@pytest.mark.parametrize("prec", ["fp64", "fp32c"])
def test_voronoi_rk4_matches_oracle(prec, gpu):
    w = configs.gaussian(level=3, delta=0.0)
    pad = 9
    vp = VorPanels(x=np.concatenate([w.xA[:, 0], np.zeros(pad)]), y=np.concatenate([w.xA[:, 1], np.zeros(pad)]),
                   z=np.concatenate([w.xA[:, 2], np.zeros(pad)]), relVort=np.concatenate([w.zetaA, np.zeros(pad)]),
                   absVort=np.zeros(w.nA + pad), area=np.concatenate([w.areaA, np.zeros(pad)]), N=w.nA)
    ctx = Context(0, prec)
    ctx.set_omega(w.omega)
    ctx.set_deltas(0.0, 0.0, 0.0)
    tke, ke = BVERK4(ctx, vp, 0.01)
    _, xA, zA, _, tke_ref, ke_ref, _ = O.bve_rk4(np.zeros((0, 3)), w.xA, w.zetaA, w.areaA, np.zeros((0, 3)),
                                                 0.01, w.omega, (0.0, 0.0, 0.0))
    got = np.stack([vp.x[:w.nA], vp.y[:w.nA], vp.z[:w.nA]], 1)
    assert rel(got - w.xA, xA - w.xA) <= TOL[prec]
    assert rel(vp.relVort[:w.nA] - w.zetaA, zA - w.zetaA) <= TOL[prec]
    assert np.all(vp.x[w.nA:] == 0)
    assert abs(tke[0] - tke_ref) <= 2 * TOL[prec] * tke_ref
    ctx.close()
