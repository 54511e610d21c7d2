"""Generate the committed fixtures of the reference's own code (tests/golden/ref_*.npz).

The reference is Fortran and no Fortran compiler is available, so its modules
run through oracle/f90, which translates the subset of Fortran 90 they use and
executes it with strict IEEE double arithmetic (see oracle/f90/__init__.py).
Every array in these fixtures was computed by the reference's own statements:
its grid generator, its initial conditions, BVERK4 / StratosphereRK4 with MPI
ranks run as threads, the three RHS sums, the Voronoi BVEVelocity and
BVERK4, finite differences of the enstrophy through its BVERK4, the file its
legacy-VTK writer writes, and its
driver programs (RHWavePanelsMPI.f90, StratospherePanels.f90 and the nine
other BVE drivers) with the rows they write to their data files. The
tests compare the C oracle, the product's host code and (on a GPU) the
product's kernels with them.

Needs the reference's sources (oracle/f90/reference.py: REFERENCE_DIR). Run from
the repository root:  python tests/golden/make_reference_fixtures.py
(about five minutes).
"""
from __future__ import annotations

import json

import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle.f90 import reference as REF  # noqa: E402

OUT = Path(__file__).resolve().parent
DT = 0.01


def _save(name, **arrays):
    np.savez_compressed(OUT / f"{name}.npz", **arrays)
    print(f"  {name}.npz")


def _flat(prefix, d):
    return {f"{prefix}_{k}": v for k, v in d.items()}


def main():
    t0 = time.time()
    g = REF.grid(3)
    _save("ref_grid_l3", **g)
    # BVERK4, parity semantics (smooth 0.05 on the divided panels), three initial conditions
    for ic, nprocs in (("rh4", 3), ("gauss", 2), ("jet", 1)):
        r = REF.bve_rk4(2, 2, DT, nprocs=nprocs, ic=ic)
        _save(f"ref_bverk4_{ic}_l2", nprocs=nprocs, dt=DT, steps=2, **_flat("initial", r["initial"]),
              **_flat("final", r["final"]), totalKE=r["totalKE"], kineticEnergy=r["kineticEnergy"])
    r = REF.bve_rk4(3, 1, DT, nprocs=4, ic="rh4")
    _save("ref_bverk4_rh4_l3", nprocs=4, dt=DT, steps=1, **_flat("initial", r["initial"]),
          **_flat("final", r["final"]), totalKE=r["totalKE"], kineticEnergy=r["kineticEnergy"])
    # StratosphereRK4 across the forcing's ramp (t = 3.95 .. 4.05)
    s = REF.strat_rk4(2, 2, 3.95, 0.05, nprocs=2)
    _save("ref_strat_l2", nprocs=2, t0=3.95, dt=0.05, steps=2, **_flat("initial", s["initial"]),
          **_flat("final", s["final"]))
    # the three RHS sums on partial ranges (one rank's share) and the Voronoi sum
    st = REF.initial_state(2, "rh4")
    xA, zA, aA, xV, xQ = st["xA"], st["zetaA"], st["areaA"], st["xV"], st["xQ"]
    dxa, dva = REF.rhs(0, None, xA, zA, aA, 37, 211)
    dxv, _ = REF.rhs(1, xV, xA, zA, aA, 11, 150)
    dxq, _ = REF.rhs(2, xQ, xA, zA, aA, 0, len(xQ))
    rng = np.random.default_rng(2)
    dy0, dz0 = rng.standard_normal(len(zA)), rng.standard_normal(len(zA))
    vor = REF.voronoi_velocity(xA[:, 0], xA[:, 1], xA[:, 2], zA, aA, 50, 300, dy=dy0, dz=dz0)
    _save("ref_rhs_l2", xA=xA, zetaA=zA, areaA=aA, xV=xV, xQ=xQ,
          active_range=np.array([37, 211]), vertex_range=np.array([11, 150]),
          active_dX=dxa, active_dVort=dva, vertex_dX=dxv, passive_dX=dxq,
          voronoi_range=np.array([50, 300]), voronoi_dy0=dy0, voronoi_dz0=dz0,
          voronoi_dx=vor[0], voronoi_dy=vor[1], voronoi_dz=vor[2], voronoi_dVort=vor[3])
    # the Voronoi solver's BVERK4 on the same generators, N_Max 10 above N, two ranks
    n, pad = len(zA), 10
    vin = {k: np.concatenate([v, np.zeros(pad)]) for k, v in
           (("x", xA[:, 0]), ("y", xA[:, 1]), ("z", xA[:, 2]), ("relVort", zA), ("area", aA))}
    vr = REF.voronoi_rk4(vin["x"], vin["y"], vin["z"], vin["relVort"], vin["area"], n, DT, 2, nprocs=2)
    _save("ref_voronoi_rk4_l2", n=n, dt=DT, steps=2, **_flat("initial", vin), **_flat("final", vr))
    # centred finite differences of J = sum zeta(T)^2 A through the reference's BVERK4 (level 1,
    # three steps): the final active vorticity for each +/- perturbation of 16 seeded entries
    _save("ref_fd_rh4_l1", **fd_inputs())
    # the file the reference's legacy-VTK writer writes (level 1, two tracers)
    v = REF.vtk_output(1)
    _save("ref_vtk_l1", **{k: (np.array(val) if k == "text" else val) for k, val in v.items()})
    # the reference's RH4 driver program (RHWavePanelsMPI.f90) on two ranks: its data-file rows
    nl = driver_namelist()
    d = REF.run_driver(2, nl)
    _save("ref_driver_rh4_l2", rows=d["rows"], nprocs=2, initNest=nl["gridInit"]["initNest"],
          dt=nl["time"]["dt"], tfinal=nl["time"]["tfinal"])
    # the reference's stratosphere driver program (StratospherePanels.f90) on two ranks
    nl = driver_namelist("strat")
    d = REF.run_driver(2, nl, which="strat")
    _save("ref_driver_strat_l2", rows=d["rows"], nprocs=2, initNest=nl["gridInit"]["initNest"],
          dt=nl["time"]["dt"], tfinal=nl["time"]["tfinal"])
    # the reference's other BVE driver programs, each from its own namelist file with the overrides
    # of other_driver_namelist, on two ranks: their data-file rows
    out = {}
    for which in OTHER_DRIVERS:
        nl = other_driver_namelist(which)
        d = REF.run_driver(2, nl, which=which)
        out[f"{which}_rows"] = d["rows"]
        out[f"{which}_namelist"] = np.array(json.dumps(nl))
    _save("ref_drivers_l2", **out)
    print(f"done in {time.time() - t0:.0f} s")


def fd_inputs(level=1, steps=3, dt=0.01, eps=1e-6, entries=16, seed=33):
    """Perturbed initial states: even entries move one panel's vorticity by +/- eps, odd entries one
    panel's position along a seeded tangent direction, renormalised to the sphere."""
    st = REF.initial_state(level, "rh4")
    xA, zA = st["xA"], st["zetaA"]
    rng = np.random.default_rng(seed)
    picks = rng.choice(len(zA), entries, replace=False)
    tangents = np.zeros((entries, 3))
    fp, fm = [], []
    for m, j in enumerate(picks):
        xp, xm, zp, zm = xA.copy(), xA.copy(), zA.copy(), zA.copy()
        if m % 2 == 0:
            zp[j] += eps
            zm[j] -= eps
        else:
            t = rng.standard_normal(3)
            t -= t.dot(xA[j]) * xA[j]
            t /= np.linalg.norm(t)
            tangents[m] = t
            xp[j] = (xA[j] + eps * t) / np.linalg.norm(xA[j] + eps * t)
            xm[j] = (xA[j] - eps * t) / np.linalg.norm(xA[j] - eps * t)
        fp.append(REF.final_active_vorticity(level, steps, dt, xp, zp))
        fm.append(REF.final_active_vorticity(level, steps, dt, xm, zm))
    return dict(xA=xA, zetaA=zA, areaA=st["areaA"], picks=picks, tangents=tangents, eps=eps,
                dt=dt, steps=steps, zeta_plus=np.array(fp), zeta_minus=np.array(fm),
                zeta_final=REF.final_active_vorticity(level, steps, dt, xA, zA))


OTHER_DRIVERS = ("gauss", "jet", "twovorts", "manyvorts", "rh2", "solidbody", "dtconv", "directrh4",
                 "zonalmean")


def other_driver_namelist(which):
    """A driver's own namelist file with the run kept small: triangular panels at level 2 (level 1
    for the dt-convergence driver, which runs five step sizes), no adaptive refinement and no
    remeshing within the run, two steps of the file's dt."""
    g = REF.read_namelist(REF.REFERENCE_DIR / REF.DRIVER_NAMELISTS[which])
    g.setdefault("gridinit", {}).update(panelkind=3, initnest=1 if which == "dtconv" else 2, amr=0,
                                        remeshinterval=1000, userelativetol=0, maxrefine=0)
    t = g.setdefault("time", {})
    t["tfinal"] = 2.5 * t["dt"]
    return g


def driver_namelist(which="rh4"):
    """Namelist groups of a driver run (the layout of the driver's .namelist file, level 2, a few
    steps, no remeshing within the run). The stratosphere run's tfinal / dt is 2.9999... in binary,
    so its floor(tfinal/dt) takes two steps, as the reference's driver does."""
    if which == "strat":
        return {"gridInit": dict(panelKind=3, initNest=2, AMR=0, remeshInterval=1000, amrTol1=1.0,
                                 amrTol2=1.0, useRelativeTol=0, maxRefine=0),
                "time": dict(dt=0.05, tfinal=0.15), "fileIO": dict(jobPrefix="strat")}
    return {"gridInit": dict(panelKind=3, initNest=2, AMR=0, remeshInterval=1000, amrTol1=1.0, amrTol2=1.0),
            "time": dict(dt=0.01, tfinal=0.03), "fileIO": dict(jobPrefix="rh4", outputDir="./")}


if __name__ == "__main__":
    main()
