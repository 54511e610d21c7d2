"""Generate the committed golden fixtures of the Biot-Savart / RK4 path.

The reference ships no golden vectors and cannot be compiled here (Fortran,
no compiler), so the fixtures are outputs of the CPU FP64 oracle
(oracle/bve_oracle.c, a line-by-line restatement of the reference loops) on
small seeded inputs. They freeze the oracle (tests/test_oracle.py checks it
reproduces them bit for bit) and give the GPU parity tests reference values
that need no oracle build where the GPU tests run.

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import oracle as O  # noqa: E402
from thesiscode_b200 import configs  # noqa: E402

OUT = Path(__file__).resolve().parent


def rh4_parity_l2():
    """Reference semantics (delta 0/0/0.05, three target classes) at level 2: the three RHS
    sums on a half range and one full BVERK4 step."""
    w = configs.rh4(level=2, parity=True, dt=0.01)
    nA = w.nA
    i0, i1 = 37, 211  # a partial [indexStart, indexEnd] range, as one MPI rank sees it
    dXA, dVA = O.active_rhs(w.xA, w.zetaA, w.areaA, i0, i1, omega=w.omega)
    dXV = O.passive_rhs(w.xV, w.xA, w.zetaA, w.areaA, 11, 150)
    dXQ = O.smooth_velocity(w.xQ, w.xA, w.zetaA, w.areaA, 0.05, 0, w.nQ)
    absV = np.zeros(w.nV) + 0.25
    xV, xA, zA, xQ, tke, ke, rel = O.bve_rk4(w.xV, w.xA, w.zetaA, w.areaA, w.xQ, w.dt, w.omega,
                                             w.deltas, absVortV=absV)
    np.savez_compressed(OUT / "rh4_parity_l2.npz", xA=w.xA, zetaA=w.zetaA, areaA=w.areaA, xV=w.xV,
                        xQ=w.xQ, omega=w.omega, dt=w.dt, deltas=np.array(w.deltas),
                        ranges=np.array([i0, i1, 11, 150]), dXA=dXA, dVA=dVA, dXV=dXV, dXQ=dXQ,
                        absV=absV, rk_xV=xV, rk_xA=xA, rk_zA=zA, rk_xQ=xQ, rk_tke=tke, rk_ke=ke,
                        rk_relV=rel, nA=nA)


def gauss_config_l3():
    """Benchmark-formula Gaussian vortex, one delta (0.01) for all targets, level 3, 2 RK4
    steps (the stage-chaining of the fused driver over more than one step)."""
    w = configs.gaussian(level=3, delta=0.01, dt=0.02)
    xV, xA, zA, xQ = w.xV, w.xA, w.zetaA, w.xQ
    tkes = []
    for _ in range(2):
        xV, xA, zA, xQ, tke, ke, _ = O.bve_rk4(xV, xA, zA, w.areaA, xQ, w.dt, w.omega, w.deltas)
        tkes.append(tke)
    np.savez_compressed(OUT / "gauss_config_l3.npz", xA=w.xA, zetaA=w.zetaA, areaA=w.areaA, xV=w.xV,
                        omega=w.omega, dt=w.dt, deltas=np.array(w.deltas), rk_xV=xV, rk_xA=xA,
                        rk_zA=zA, rk_tke=np.array(tkes), rk_ke=ke)


def voronoi_l2():
    """BVEVelocity on SoA arrays with unused N_Max slots (vort = area = 0)."""
    w = configs.rh4(level=2, parity=False, delta=0.0)
    n = w.nA
    pad = 17
    x = np.concatenate([w.xA[:, 0], np.zeros(pad)])
    y = np.concatenate([w.xA[:, 1], np.zeros(pad)])
    z = np.concatenate([w.xA[:, 2], np.zeros(pad)])
    vort = np.concatenate([w.zetaA, np.zeros(pad)])
    area = np.concatenate([w.areaA, np.zeros(pad)])
    dx, dy, dz, dV = O.voronoi_velocity(x, y, z, vort, area, 0, n, omega=w.omega)
    np.savez_compressed(OUT / "voronoi_l2.npz", x=x, y=y, z=z, vort=vort, area=area, n=n,
                        omega=w.omega, dx=dx, dy=dy, dz=dz, dV=dV)


if __name__ == "__main__":
    rh4_parity_l2()
    gauss_config_l3()
    voronoi_l2()
    for p in sorted(OUT.glob("*.npz")):
        print(p.name, p.stat().st_size)
