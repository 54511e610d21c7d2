"""The Fortran drop-in module itself, run against the library on the GPU.

thesiscode_b200/fortran/PanelVelocityCUDA.f90 is what a reference driver
compiles in place of PanelVelocityParallelModule. Neither machine has a
Fortran compiler, so it runs through oracle/f90 (the translator of the
Fortran 90 subset that also runs the reference's own modules) on top of the
reference's ParticlesEdgesPanels / TracerAndVorticityDistributions modules,
its BIND(C) interface calls going to libthesiscode_b200.so through ctypes
and its MPI_ALLGATHERV to an in-process exchange between ranks run as
threads (each rank its own library context on this GPU; no kernel of one
rank waits for another). The reference's grid and initial condition are
built inside the same program, exactly as a driver does before calling
BVERK4, and the results are compared with the reference's own BVERK4 /
StratosphereRK4 (tests/golden/ref_*.npz, PanelVelocityParallel.f90:435-919).

Tolerances as in tests/test_reference_gpu.py: FP64 1e-12, FP32C 5e-7 (level
<= 3), relative to the largest displacement (vorticity change).
"""
from pathlib import Path

import numpy as np
import pytest

from oracle.f90 import reference as REF
from thesiscode_b200 import _native as N

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not REF.shim_built(),
                                 reason="the drop-in's translation is built by __graft_entry__.build() "
                                        "where the reference's sources are present")]
GOLDEN = Path(__file__).resolve().parent / "golden"
TOL = {False: 1e-12, True: 5e-7}


def _load(name):
    return dict(np.load(GOLDEN / f"{name}.npz"))


def _state(f, prefix):
    n = len(prefix) + 1
    return {k[n:]: v for k, v in f.items() if k.startswith(prefix + "_")}


def rel_err(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _check(run, f, tol, keys=("xA", "xV", "xQ", "zetaA")):
    s0, s1 = _state(f, "initial"), _state(f, "final")
    for k, v in s0.items():  # the driver-side inputs are the reference's, bit for bit
        assert np.array_equal(run["initial"][k], v), k
    for k in keys:
        assert rel_err(run["final"][k] - s0[k], s1[k] - s0[k]) <= tol, k
    assert rel_err(run["final"]["relVortV"], s1["relVortV"]) <= tol  # :651


@pytest.mark.parametrize("fp32c", [False, True])
def test_dropin_bverk4_one_rank(fp32c, gpu):
    f = _load("ref_bverk4_rh4_l2")
    run = REF.shim_bve_rk4(N.LIB_PATH, 2, int(f["steps"]), float(f["dt"]), nprocs=1, fp32c=fp32c)
    _check(run, f, TOL[fp32c])
    assert rel_err(run["totalKE"], f["totalKE"]) <= 2 * TOL[fp32c]
    assert rel_err(run["kineticEnergy"], f["kineticEnergy"]) <= 2 * TOL[fp32c]


@pytest.mark.parametrize("name,level,nprocs", [("ref_bverk4_rh4_l2", 2, 3), ("ref_bverk4_rh4_l3", 3, 4)])
def test_dropin_bverk4_sharded_ranks(name, level, nprocs, gpu):
    """numProcs > 1: each rank steps its LoadBalance rows (ragged at level 3: 642 particles on 4
    ranks) and exchanges source rows with MPI_ALLGATHERV after every stage; all ranks end with
    the same state, the reference's."""
    f = _load(name)
    run = REF.shim_bve_rk4(N.LIB_PATH, level, int(f["steps"]), float(f["dt"]), nprocs=nprocs)
    _check(run, f, TOL[False])
    assert rel_err(run["totalKE"], f["totalKE"]) <= 2 * TOL[False]
    for r in run["ranks"][1:]:
        for k, v in run["final"].items():
            assert np.array_equal(r["final"][k], v), k
        assert np.array_equal(r["totalKE"], run["totalKE"])


@pytest.mark.parametrize("fp32c", [False, True])
def test_dropin_stratosphere_rk4(fp32c, gpu):
    f = _load("ref_strat_l2")
    run = REF.shim_strat_rk4(N.LIB_PATH, 2, int(f["steps"]), float(f["t0"]), float(f["dt"]),
                             nprocs=2, fp32c=fp32c)
    _check(run, f, TOL[fp32c], keys=("xA", "xV", "xQ"))
    assert rel_err(run["final"]["zetaA"], _state(f, "final")["zetaA"]) <= TOL[fp32c]


def _driver_namelist(f):
    return {"gridInit": dict(panelKind=3, initNest=int(f["initNest"]), AMR=0, remeshInterval=1000,
                             amrTol1=1.0, amrTol2=1.0),
            "time": dict(dt=float(f["dt"]), tfinal=float(f["tfinal"])),
            "fileIO": dict(jobPrefix="rh4", outputDir="./")}


@pytest.mark.skipif(not REF.driver_built(), reason="the driver's translation is built by "
                    "__graft_entry__.build() where the reference's sources are present")
@pytest.mark.parametrize("nprocs,fp32c", [(1, False), (2, False), (1, True)])
def test_reference_driver_with_its_use_line_switched(nprocs, fp32c, gpu):
    """The reference's RH4 driver program (RHWavePanelsMPI.f90) unmodified except for
    `use PanelVelocityParallelModule` -> `use PanelVelocityCUDAModule`: namelist in, grid and
    initial condition built by the driver, BVERK4 each step on the GPU, and the rows it writes to
    its data file (totalKE, enstrophy, relVort l1 / l2 / linf error against the steady wave) equal
    those of the unmodified driver (tests/golden/ref_driver_rh4_l2.npz). The error norms are
    differences of vorticities: compared to an absolute 10x the vorticity tolerance."""
    f = _load("ref_driver_rh4_l2")
    run = REF.run_driver(nprocs, _driver_namelist(f), cuda=True, lib_path=N.LIB_PATH, fp32c=fp32c)
    rows, ref = run["rows"], f["rows"]
    assert rows.shape == ref.shape
    tol = TOL[fp32c]
    assert rel_err(rows[:, 0], ref[:, 0]) <= 2 * tol      # totalKE
    assert rel_err(rows[:, 1], ref[:, 1]) <= 2 * tol      # enstrophy
    assert np.abs(rows[:, 2:] - ref[:, 2:]).max() <= 10 * tol


@pytest.mark.skipif(not REF.driver_built("strat"), reason="the driver's translation is built by "
                    "__graft_entry__.build() where the reference's sources are present")
@pytest.mark.parametrize("nprocs,fp32c", [(1, False), (2, False), (1, True)])
def test_reference_stratosphere_driver_with_its_use_line_switched(nprocs, fp32c, gpu):
    """The reference's forced-model driver (StratospherePanels.f90) with only its `use` line
    switched to the drop-in module: StratosphereRK4 each step on the GPU; its data-file rows
    (totalKE, enstrophy per step) equal the unmodified driver's (tests/golden/ref_driver_strat_l2.npz)."""
    f = _load("ref_driver_strat_l2")
    nl = {"gridInit": dict(panelKind=3, initNest=int(f["initNest"]), AMR=0, remeshInterval=1000,
                           amrTol1=1.0, amrTol2=1.0, useRelativeTol=0, maxRefine=0),
          "time": dict(dt=float(f["dt"]), tfinal=float(f["tfinal"])), "fileIO": dict(jobPrefix="strat")}
    run = REF.run_driver(nprocs, nl, cuda=True, lib_path=N.LIB_PATH, fp32c=fp32c, which="strat")
    rows, ref = run["rows"], f["rows"]
    assert rows.shape == ref.shape
    tol = TOL[fp32c]
    assert rel_err(rows[1:, 0], ref[1:, 0]) <= 2 * tol     # totalKE (row 0 is the unset initial 0)
    assert rel_err(rows[:, 1], ref[:, 1]) <= 2 * tol       # enstrophy


OTHER_DRIVERS = ("gauss", "jet", "twovorts", "manyvorts", "rh2", "solidbody", "dtconv", "directrh4",
                 "zonalmean")


@pytest.mark.parametrize("which", OTHER_DRIVERS)
def test_other_reference_drivers_with_their_use_line_switched(which, gpu):
    """Every other BVE driver of the reference (Gaussian vortex, jet, two and many vortices,
    Rossby-Haurwitz 2, solid body, the dt-convergence study that resets the RK4 state for each of
    its step sizes, the direct RH4 run, the zonal mean), each from its own namelist file kept
    small (tests/golden/make_reference_fixtures.py), with only its `use` line switched to the
    drop-in module, on 2 ranks in FP64: the rows it writes to its data file equal those the
    unmodified driver writes (tests/golden/ref_drivers_l2.npz), to 1e-10 relative or 1e-12
    absolute (some columns are error norms of a few 1e-10, differences of two runs)."""
    import json

    if not REF.driver_built(which):
        pytest.skip("the driver's translation is built by __graft_entry__.build() where the "
                    "reference's sources are present")
    f = _load("ref_drivers_l2")
    nl = json.loads(str(f[f"{which}_namelist"]))
    run = REF.run_driver(2, nl, cuda=True, lib_path=N.LIB_PATH, which=which)
    ref = f[f"{which}_rows"]
    assert run["rows"].shape == ref.shape
    assert np.allclose(run["rows"], ref, rtol=1e-10, atol=1e-12), np.abs(run["rows"] - ref).max()
