"""The reference's hot path run from its own Fortran source (ThesisCode, free-form .f90).

TEST INFRASTRUCTURE ONLY: used by tests/ and tests/golden/make_reference_fixtures.py
to pin the C oracle to the reference's code. Needs the reference's sources
(REFERENCE_DIR, default the checkout this build was given); where they are
absent, available() is False and the committed fixtures stand in for them.

What runs, all of it the reference's own statements translated by
oracle/f90 (nothing restated here):
  * NewGrid -> InitIcosTriGrid / DivideTriPanel / TriPanelArea
    (ParticlesEdgesPanels2.f90:362-397,419-1090,1727-1802), the grid;
  * InitRH4WavePanels, InitGaussianVortexPanels, InitJetPanels
    (TracerAndVorticityDistributions.f90:142-174,243-304,737-790,793-812), the initial vorticity;
  * InitializeMPIRK4 / LoadBalance / BVERK4 / StratosphereRK4 and the three RHS sums
    (PanelVelocityParallel.f90:126-213,435-919,1287-1412), with MPI ranks as threads and
    MPI_BCAST as an in-process broadcast;
  * BVEVelocity and the RK4 step of BVERK4 of the Voronoi solver
    (VoronoiVelocityParallel.f90:252-515);
  * the legacy-VTK writer vtkOutputUnif (ParticlesEdgesPanels2.f90:2116-2237), its formatted
    WRITEs collected as text.
Logger and OutputWriter procedures (logging and file output) are replaced by no-ops, and so is
the STRIPACK Delaunay / Voronoi rebuild at the end of the Voronoi BVERK4.

The same translator also runs this repository's Fortran drop-in module
(thesiscode_b200/fortran/PanelVelocityCUDA.f90) on top of the reference's
modules, its BIND(C) interfaces calling the library through ctypes: the module
a Fortran driver would compile, executed against the real GPU library (no
Fortran compiler exists on either machine). build_programs() writes both
translations to oracle/_ref/ (a build output, git-ignored, carried to the GPU
machine like the library), from where they load when the sources are absent.
"""
from __future__ import annotations

import ctypes
import os
import threading
import time
from functools import lru_cache
from pathlib import Path

import numpy as np

from . import Runner, load, rt

REFERENCE_DIR = Path(os.environ.get("TC_REFERENCE_DIR", "/root/reference"))
ROOT = Path(__file__).resolve().parents[2]
BUILD_DIR = ROOT / "oracle" / "_ref"
SHIM = ROOT / "thesiscode_b200" / "fortran" / "PanelVelocityCUDA.f90"

FILES = ("NumberKinds.f90", "SphereGeom.f90", "OutputWriter.f90", "Logger.f90", "IntegerList.f90",
         "ParticlesEdgesPanels2.f90", "VoronoiPanels.f90", "STRIPACK.f90",
         "TracerAndVorticityDistributions.f90", "PanelVelocityParallel.f90",
         "VoronoiVelocityParallel.f90")

PVP = "panelvelocityparallelmodule"
PEP = "particlesedgespanelsmodule"
TVD = "tracerandvorticitydistributionmodule"
VVP = "voronoivelocityparallelmodule"
PVC = "panelvelocitycudamodule"
PVS = "panelvelocityserialmodule"

ENTRY = [(PVP, p) for p in ("bverk4", "stratosphererk4", "initializempirk4", "finalizempirk4",
                            "setsmooth", "bveactiverhs", "bvepassiverhs", "bvesmoothvelocity")] + \
        [(PEP, "newgrid"), (TVD, "setomega"), (TVD, "initrh4wavepanels"),
         (TVD, "initgaussianvortexpanels"), (TVD, "initjetpanels"), (TVD, "initstratosphere"),
         (VVP, "bvevelocity"), (VVP, "bverk4"), (VVP, "initializempirk4"), (VVP, "finalizempirk4"),
         (PEP, "vtkoutputunif")]
VPM = "voronoipanelsmodule"

SHIM_ENTRY = [(PVC, p) for p in ("bverk4", "stratosphererk4", "initializempirk4", "finalizempirk4",
                                  "setsmooth", "getsmooth", "setprecisioncuda", "resetrk4",
                                  "loadbalance")] + \
             [(PEP, "newgrid"), (TVD, "setomega"), (TVD, "initrh4wavepanels"),
              (TVD, "initgaussianvortexpanels"), (TVD, "initjetpanels"), (TVD, "initstratosphere")]

# mpif.h stand-in: only the names the modules use; the values are handles the host procedures
# receive and never interpret (MPI_SUCCESS is 0, as in every MPI)
MPIF = {"mpi_status_size": 6, "mpi_double_precision": 17, "mpi_integer": 7, "mpi_comm_world": 0,
        "mpi_real": 13, "mpi_sum": 1, "mpi_logical": 6, "mpi_max": 2, "mpi_min": 3, "mpi_success": 0}
HOST_PROCS = {"mpi_bcast", "mpi_barrier", "mpi_allgatherv", "mpi_init", "mpi_finalize",
              "mpi_comm_size", "mpi_comm_rank", "mpi_wtime"}

# the reference's driver programs run here: (source file, program name); each is switched to the
# drop-in module by its one `use PanelVelocityParallelModule` line
DRIVERS = {"rh4": ("RHWavePanelsMPI.f90", "rhwavepanelsmpi"),
           "strat": ("StratospherePanels.f90", "stratospherepanels"),
           "gauss": ("GaussVort.f90", "gaussianvortex"),
           "jet": ("JetPanels.f90", "jetpanels"),
           "twovorts": ("TwoVortsPanels.f90", "twovortices"),
           "manyvorts": ("ManyVortsPanels.f90", "manyvortspanels"),
           "rh2": ("RH2Panels.f90", "rh2wavepanels"),
           "solidbody": ("solidBody.f90", "solidbody"),
           "dtconv": ("BVEDeltaTConv.f90", "bvedeltatconv"),
           "directrh4": ("DirectRH4Panels.f90", "directrhwave"),
           "zonalmean": ("ZonalMeanPanels.f90", "zonalmean")}
# the namelist file each driver opens
DRIVER_NAMELISTS = {"rh4": "RHWavePanels.namelist", "strat": "StratospherePanels.namelist",
                    "gauss": "GaussVortPanels.namelist", "jet": "JetPanels.namelist",
                    "twovorts": "TwoVorts.namelist", "manyvorts": "ManyVortsPanels.namelist",
                    "rh2": "RH2Panels.namelist", "solidbody": "SolidBody.namelist",
                    "dtconv": "BVEDTConv.namelist", "directrh4": "RHWavePanels.namelist",
                    "zonalmean": "ZonalMeanPanels.namelist"}
DRIVER, DRV = DRIVERS["rh4"]
DRIVER_ALIASES = {"panelvelocityparallelmodule": PVC}

TRI_PANEL, BVE_SOLVER = 3, 61


def available() -> bool:
    return all((REFERENCE_DIR / f).is_file() for f in FILES)


def _stub(mod, proc):
    """Logging and file output are no-ops; so is the Delaunay / Voronoi rebuild (STRIPACK) that the
    Voronoi solver's BVERK4 calls after its step (VoronoiVelocityParallel.f90:480-482): it changes
    the mesh for the next step, not the step's positions, vorticity or kinetic energy."""
    if mod == "voronoipanelsmodule" and proc in ("normalizegrid", "delaunaytri", "voronoigrid"):
        return True
    return mod == "outputwritermodule" or (mod == "loggermodule" and proc != "getlogginglevel")


def _driver_stub(mod, proc):
    """The driver's run leaves out remeshing (out of scope; raises if reached) and VTK / statistics
    output (no-ops)."""
    if mod == "refineremeshmodule":
        return "raise"
    if mod == PEP and (proc.startswith("vtkoutput") or proc.startswith("print")):
        return True
    return _stub(mod, proc)


def _program(name, files, entry, stubs=_stub, aliases=None):
    """The translation: generated from the sources where they are, else loaded from its build."""
    if available():
        return Runner(files, entry, includes={"mpif.h": MPIF}, host_procs=HOST_PROCS, stubs=stubs,
                      use_aliases=aliases)
    built = BUILD_DIR / name
    if built.is_file():
        return load(built)
    raise FileNotFoundError(f"neither the reference's sources ({REFERENCE_DIR}) nor {built} exist")


@lru_cache(maxsize=1)
def runner():
    """The reference's modules."""
    return _program("f90_reference.py", [REFERENCE_DIR / f for f in FILES], ENTRY)


@lru_cache(maxsize=1)
def shim_runner():
    """The Fortran drop-in module with the reference's modules it uses."""
    return _program("f90_shim.py", [REFERENCE_DIR / f for f in FILES] + [SHIM], SHIM_ENTRY)


def _driver_file(which, cuda):
    return f"f90_driver{'' if which == 'rh4' else '_' + which}{'_cuda' if cuda else ''}.py"


@lru_cache(maxsize=4)
def driver_runner(cuda: bool, which: str = "rh4"):
    """A driver program of the reference (DRIVERS), with `use PanelVelocityParallelModule` as
    written (cuda False) or switched to the drop-in module (cuda True)."""
    src, prog = DRIVERS[which]
    files = [REFERENCE_DIR / f for f in FILES] + [REFERENCE_DIR / "RefineRemesh.f90", REFERENCE_DIR / src]
    if cuda:
        return _program(_driver_file(which, True), files + [SHIM], [(prog, "main"), (PVC, "setprecisioncuda")],
                        _driver_stub, DRIVER_ALIASES)
    return _program(_driver_file(which, False), files, [(prog, "main")], _driver_stub)


@lru_cache(maxsize=1)
def serial_runner():
    """The reference's serial twin of the RK4 module (PanelVelocitySerial.f90)."""
    return _program("f90_serial.py", [REFERENCE_DIR / f for f in FILES] +
                    [REFERENCE_DIR / "PanelVelocitySerial.f90"],
                    [(PVS, "bverk4"), (PVS, "resetrk4"), (PEP, "newgrid"), (TVD, "initrh4wavepanels"),
                     (TVD, "initgaussianvortexpanels"), (TVD, "initjetpanels")])


def serial_bve_rk4(level, steps, dt, ic="rh4") -> dict:
    """BVERK4 of PanelVelocitySerial.f90:272-425 (one process, smooth 0.05, Omega 2 pi) from the
    reference's grid and initial condition."""
    inst = serial_runner().instance()
    p, _, q = new_grid(inst, level)
    _init(inst, ic, p, q)
    s0 = state(p, q)
    tke = []
    for _ in range(steps):
        inst.proc(PVS, "bverk4")(p, q, dt)
        tke.append(float(inst.mod(PVS).totalke))
    return dict(initial=s0, final=state(p, q), totalKE=np.array(tke),
                kineticEnergy=inst.mod(PVS).kineticenergy.a.copy())


def shim_built() -> bool:
    return available() or (BUILD_DIR / "f90_shim.py").is_file()


def driver_built(which: str = "rh4") -> bool:
    return available() or (BUILD_DIR / _driver_file(which, True)).is_file()


def build_programs() -> list:
    """Write the translations to oracle/_ref/ (where the reference's sources are present)."""
    if not available():
        return []
    BUILD_DIR.mkdir(parents=True, exist_ok=True)
    out = []
    for name, r, extra in (("f90_reference.py", runner(), ""),
                           ("f90_shim.py", shim_runner(), ", thesiscode_b200/fortran/PanelVelocityCUDA.f90"),
                           *((_driver_file(w, True), driver_runner(True, w),
                              f", RefineRemesh.f90, {DRIVERS[w][0]} (use switched to the drop-in), "
                              "thesiscode_b200/fortran/PanelVelocityCUDA.f90") for w in DRIVERS)):
        r.save(BUILD_DIR / name, note=f"sources: {', '.join(FILES)}{extra}")
        out.append(BUILD_DIR / name)
    return out


class _World:
    """In-process MPI_COMM_WORLD for ranks run as threads."""

    def __init__(self, n):
        self.bar = threading.Barrier(n, timeout=600)
        self.slot = None

    def bcast(self, rank, buf, count, datatype, root, comm, ierr):
        a = buf.a if isinstance(buf, rt.FArr) else None
        if a is None or a.size != count:
            raise ValueError(f"MPI_BCAST of {count} values on a buffer of {None if a is None else a.size}")
        if rank == root:
            self.slot = a.copy()
        self.bar.wait()
        if rank != root:
            a[...] = self.slot
        self.bar.wait()

    def barrier(self):
        self.bar.wait()

    def allgatherv(self, rank, send, scount, stype, recv, counts, displs, rtype, comm, ierr):
        if rank == 0:
            self.slot = {}
        self.bar.wait()
        self.slot[rank] = np.array(send.a.reshape(-1, order="F")[:int(scount)])
        self.bar.wait()
        flat = recv.a.reshape(-1, order="F")
        for j in range(counts.a.size):
            c, d = int(counts.a[j]), int(displs.a[j])
            flat[d:d + c] = self.slot[j][:c]
        if not np.shares_memory(flat, recv.a):
            raise ValueError("MPI_ALLGATHERV receive buffer is not contiguous")
        self.bar.wait()


def _ranks(nprocs, body, program=None, host=None):
    """Run body(instance, rank) on nprocs thread ranks; returns the per-rank results. host: extra
    host entries, or a function of the rank giving them."""
    r = program or runner()
    world = _World(nprocs)
    out, errs = [None] * nprocs, []

    def main(rank):
        try:
            extra = host(rank) if callable(host) else (host or {})
            inst = r.instance(host={"mpi_bcast": lambda *a: world.bcast(rank, *a),
                                    "mpi_barrier": lambda *a: world.barrier(),
                                    "mpi_allgatherv": lambda *a: world.allgatherv(rank, *a),
                                    "mpi_init": lambda *a: None,
                                    "mpi_finalize": lambda *a: None,
                                    "mpi_comm_size": lambda comm, n, ierr: (rt.NO, nprocs, 0),
                                    "mpi_comm_rank": lambda comm, k, ierr: (rt.NO, rank, 0),
                                    "mpi_wtime": time.perf_counter,
                                    **extra})
            out[rank] = body(inst, rank)
        except BaseException as e:  # noqa: BLE001 - re-raised below
            errs.append(e)
            world.bar.abort()

    threads = [threading.Thread(target=main, args=(k,)) for k in range(nprocs)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    if errs:
        raise errs[0]
    return out


def new_grid(inst, level, n_tracer=1):
    g = inst.proc(PEP, "newgrid")(None, None, None, TRI_PANEL, level, 0, n_tracer, BVE_SOLVER)
    return g[0], g[1], g[2]


def grid(level) -> dict:
    """The reference's icosahedral grid: the arrays of oracle.icos_grid (0-based tables)."""
    inst = runner().instance()
    p, _, q = new_grid(inst, level)
    n, m = p.n, q.n
    return dict(particles_x=p.x.a[:, :n].T.copy(), particles_x0=p.x0.a[:, :n].T.copy(),
                panels_x=q.x.a[:, :m].T.copy(), panels_x0=q.x0.a[:, :m].T.copy(),
                panels_area=q.area.a[:m].copy(),
                panels_has_children=q.haschildren.a[:m].astype(np.int32),
                panels_vertices=(q.vertices.a[:, :m].T - 1).astype(np.int32),
                panels_nest=q.nest.a[:m].astype(np.int32),
                panels_children=(q.children.a[:, :m].T - 1).astype(np.int32))


def _init(inst, ic, p, q):
    if ic == "rh4":
        inst.proc(TVD, "initrh4wavepanels")(p, q)
    elif ic == "gauss":
        inst.proc(TVD, "initgaussianvortexpanels")(p, q)
    elif ic == "jet":
        inst.proc(TVD, "initjetpanels")(p, q, np.pi / 4.0, 12.0, 0.025, 12)
    elif ic == "strat":
        inst.proc(TVD, "initstratosphere")(p, q)
    else:
        raise ValueError(ic)


def state(p, q) -> dict:
    """Particles and panels as arrays: the gathered classes of the RK4 step in index order."""
    n, m = p.n, q.n
    hc = q.haschildren.a[:m].astype(bool)
    act, pas = np.nonzero(~hc)[0], np.nonzero(hc)[0]
    return dict(xV=p.x.a[:, :n].T.copy(), relVortV=p.relvort.a[:n].copy(), absVortV=p.absvort.a[:n].copy(),
                xA=q.x.a[:, act].T.copy(), zetaA=q.relvort.a[act].copy(), absVortA=q.absvort.a[act].copy(),
                areaA=q.area.a[act].copy(), xQ=q.x.a[:, pas].T.copy())


def initial_state(level, ic="rh4") -> dict:
    inst = runner().instance()
    p, _, q = new_grid(inst, level)
    _init(inst, ic, p, q)
    return state(p, q)


def bve_rk4(level, steps, dt, nprocs=1, ic="rh4", smooth=0.05, omega=2 * np.pi) -> dict:
    """BVERK4 (PanelVelocityParallel.f90:435-658) for `steps` steps on nprocs thread ranks, from
    the reference's grid and initial condition. Returns the initial and final states, the
    totalKE of every step and each rank's final state (all ranks must agree)."""
    def body(inst, rank):
        inst.proc(TVD, "setomega")(omega)
        inst.proc(PVP, "setsmooth")(smooth)
        p, _, q = new_grid(inst, level)
        _init(inst, ic, p, q)
        s0 = state(p, q)
        inst.proc(PVP, "initializempirk4")(p, q, rank, nprocs)
        tke = []
        for _ in range(steps):
            inst.proc(PVP, "bverk4")(p, q, dt, rank, nprocs)
            tke.append(float(inst.mod(PVP).totalke))
        ke = inst.mod(PVP).kineticenergy.a.copy()
        inst.proc(PVP, "finalizempirk4")()
        return s0, state(p, q), tke, ke

    res = _ranks(nprocs, body)
    s0, s1, tke, ke = res[0]
    for _, s, t, _k in res[1:]:
        if t != tke or any(not np.array_equal(s[k], s1[k]) for k in s1):
            raise AssertionError("ranks disagree after BVERK4")
    return dict(initial=s0, final=s1, totalKE=np.array(tke), kineticEnergy=ke)


def final_active_vorticity(level, steps, dt, xA, zetaA, ic="rh4", omega=2 * np.pi) -> np.ndarray:
    """BVERK4 (one rank) from the reference's grid and initial condition with the active panels'
    positions and vorticity replaced by xA, zetaA (the inputs of a finite difference); returns the
    active panels' vorticity after `steps` steps."""
    def body(inst, rank):
        inst.proc(TVD, "setomega")(omega)
        p, _, q = new_grid(inst, level)
        _init(inst, ic, p, q)
        act = np.nonzero(~q.haschildren.a[:q.n].astype(bool))[0]
        q.x.a[:, act] = np.asarray(xA).T
        q.relvort.a[act] = zetaA
        inst.proc(PVP, "initializempirk4")(p, q, rank, 1)
        for _ in range(steps):
            inst.proc(PVP, "bverk4")(p, q, dt, rank, 1)
        out = q.relvort.a[act].copy()
        inst.proc(PVP, "finalizempirk4")()
        return out

    return _ranks(1, body)[0]


def strat_rk4(level, steps, t0, dt, nprocs=1, smooth=0.05, omega=2 * np.pi) -> dict:
    """StratosphereRK4 (PanelVelocityParallel.f90:661-919): the forced model's step, from the
    reference's stratosphere initial condition (InitStratosphere)."""
    def body(inst, rank):
        inst.proc(TVD, "setomega")(omega)
        inst.proc(PVP, "setsmooth")(smooth)
        p, _, q = new_grid(inst, level)
        _init(inst, "strat", p, q)
        s0 = state(p, q)
        inst.proc(PVP, "initializempirk4")(p, q, rank, nprocs)
        t = t0
        for _ in range(steps):
            inst.proc(PVP, "stratosphererk4")(p, q, t, dt, rank, nprocs)
            t = t + dt
        inst.proc(PVP, "finalizempirk4")()
        return s0, state(p, q)

    res = _ranks(nprocs, body)
    s0, s1 = res[0]
    for _, s in res[1:]:
        if any(not np.array_equal(s[k], s1[k]) for k in s1):
            raise AssertionError("ranks disagree after StratosphereRK4")
    return dict(initial=s0, final=s1)


def _f2(a):
    return rt.FArr(np.asfortranarray(np.asarray(a, dtype=np.float64).T))


def _f1(a):
    return rt.FArr(np.array(a, dtype=np.float64))


def rhs(cls, X, x, vort, area, i0, i1, smooth=0.05, omega=2 * np.pi):
    """One of BVEActiveRHS (cls 0), BVEPassiveRHS (1), BVESmoothVelocity (2) over the 0-based
    half-open row range [i0, i1) (Fortran indexStart = i0 + 1, indexEnd = i1); returns dX (m, 3)
    and, for the active sum, dVort."""
    inst = runner().instance()
    inst.proc(TVD, "setomega")(omega)
    inst.proc(PVP, "setsmooth")(smooth)
    n = len(vort)
    if cls == 0:
        dx, dv = rt.FArr(np.zeros((3, n), order="F")), rt.FArr(np.zeros(n))
        inst.proc(PVP, "bveactiverhs")(dx, dv, _f2(x), _f1(vort), _f1(area), i0 + 1, i1)
        return dx.a.T.copy(), dv.a.copy()
    m = len(X)
    dx = rt.FArr(np.zeros((3, m), order="F"))
    name = "bvepassiverhs" if cls == 1 else "bvesmoothvelocity"
    inst.proc(PVP, name)(dx, _f2(X), _f2(x), _f1(vort), _f1(area), i0 + 1, i1)
    return dx.a.T.copy(), None


def voronoi_velocity(x, y, z, vort, area, i0, i1, omega=2 * np.pi, dy=None, dz=None):
    """BVEVelocity of the Voronoi solver (VoronoiVelocityParallel.f90:487-515) over rows [i0, i1):
    (dx, dy, dz, dVort). dy and dz start from the given arrays (the routine zeroes dx only)."""
    inst = runner().instance()
    inst.proc(TVD, "setomega")(omega)
    n = len(x)
    out = [rt.FArr(np.zeros(n)), _f1(np.zeros(n) if dy is None else dy),
           _f1(np.zeros(n) if dz is None else dz), rt.FArr(np.zeros(n))]
    inst.proc(VVP, "bvevelocity")(*out, _f1(x), _f1(y), _f1(z), _f1(vort), _f1(area), i0 + 1, i1)
    return tuple(o.a.copy() for o in out)


def voronoi_rk4(x, y, z, relvort, area, n, dt, steps, nprocs=1, omega=2 * np.pi) -> dict:
    """BVERK4 of the Voronoi solver (VoronoiVelocityParallel.f90:300-483) on nprocs thread ranks:
    generators 1..n of arrays of length N_Max = len(x) (the sums run over all N_Max slots, the
    unused ones carrying zero vorticity and area). Returns the first n positions and relVort after
    `steps` steps and totalKE of each step."""
    def body(inst, rank):
        inst.proc(TVD, "setomega")(omega)
        vp = inst.new(VPM, "vorpanels")
        nmax = len(x)
        vp.x, vp.y, vp.z = _f1(x), _f1(y), _f1(z)
        vp.x0, vp.y0, vp.z0 = _f1(x), _f1(y), _f1(z)
        vp.relvort, vp.area = _f1(relvort), _f1(area)
        vp.absvort = _f1(np.asarray(relvort) + 2.0 * omega * np.asarray(z))
        vp.n, vp.n_max = int(n), int(nmax)
        inst.proc(VVP, "initializempirk4")(int(n), rank, nprocs)
        tke = []
        for _ in range(steps):
            inst.proc(VVP, "bverk4")(vp, dt, rank, nprocs)
            tke.append(float(inst.mod(VVP).totalke))
        inst.proc(VVP, "finalizempirk4")()
        return dict(x=vp.x.a[:n].copy(), y=vp.y.a[:n].copy(), z=vp.z.a[:n].copy(),
                    relVort=vp.relvort.a[:n].copy(), totalKE=np.array(tke))

    res = _ranks(nprocs, body)
    for r in res[1:]:
        if any(not np.array_equal(r[k], res[0][k]) for k in res[0]):
            raise AssertionError("ranks disagree after the Voronoi BVERK4")
    return res[0]


def vtk_output(level, ic="rh4", n_tracer=2) -> dict:
    """vtkOutputUnif (ParticlesEdgesPanels2.f90:2116-2237) on the reference's grid with its
    initial condition and seeded tracer values: the text of the file it writes, and the arrays it
    was written from (particles then panels, every panel)."""
    files, records = {}, {}
    host = {"__open__": lambda unit, name: files.__setitem__(int(unit), name),
            "__record__": lambda unit, recs: records.setdefault(int(unit), []).extend(recs),
            "__close__": lambda unit: None}
    inst = runner().instance(host=host)
    p, _, q = new_grid(inst, level, n_tracer)
    _init(inst, ic, p, q)
    rng = np.random.default_rng(level)
    n, m = p.n, q.n
    p.tracer.a[:n, :] = rng.standard_normal((n, n_tracer))
    q.tracer.a[:m, :] = rng.standard_normal((m, n_tracer))
    inst.proc(PEP, "vtkoutputunif")(p, q, "grid.vtk")
    (unit,) = [u for u, name in files.items() if name == "grid.vtk"]
    return dict(text="\n".join(records[unit]) + "\n",
                particles_relVort=p.relvort.a[:n].copy(), particles_absVort=p.absvort.a[:n].copy(),
                particles_tracer=p.tracer.a[:n, :].copy(), panels_relVort=q.relvort.a[:m].copy(),
                panels_absVort=q.absvort.a[:m].copy(), panels_tracer=q.tracer.a[:m, :].copy())


# ----------------------------------------------------------------------------- the drop-in
def _lib(lib_path):
    return ctypes.CDLL(str(lib_path))


def shim_bve_rk4(lib_path, level, steps, dt, nprocs=1, fp32c=False, ic="rh4", smooth=0.05,
                 omega=2 * np.pi) -> dict:
    """The drop-in module's BVERK4 (PanelVelocityCUDA.f90) on nprocs thread ranks, on the
    reference's grid and initial condition, with the library at lib_path doing the step (one
    context per rank; numProcs > 1 takes the sharded path with MPI_ALLGATHERV)."""
    lib = _lib(lib_path)

    def body(inst, rank):
        inst.proc(TVD, "setomega")(omega)
        inst.proc(PVC, "setsmooth")(smooth)
        inst.proc(PVC, "setprecisioncuda")(bool(fp32c))
        p, _, q = new_grid(inst, level)
        _init(inst, ic, p, q)
        s0 = state(p, q)
        inst.proc(PVC, "initializempirk4")(p, q, rank, nprocs)
        tke = []
        for _ in range(steps):
            inst.proc(PVC, "bverk4")(p, q, dt, rank, nprocs)
            tke.append(float(inst.mod(PVC).totalke))
        ke = inst.mod(PVC).kineticenergy.a.copy()
        inst.proc(PVC, "finalizempirk4")()
        return s0, state(p, q), tke, ke

    res = _ranks(nprocs, body, shim_runner(), {"__cdll__": lib})
    s0, s1, tke, ke = res[0]
    return dict(initial=s0, final=s1, totalKE=np.array(tke), kineticEnergy=ke,
                ranks=[dict(final=r[1], totalKE=np.array(r[2])) for r in res])


def shim_strat_rk4(lib_path, level, steps, t0, dt, nprocs=1, fp32c=False, smooth=0.05,
                   omega=2 * np.pi) -> dict:
    """The drop-in module's StratosphereRK4 on nprocs thread ranks (every rank runs the step)."""
    lib = _lib(lib_path)

    def body(inst, rank):
        inst.proc(TVD, "setomega")(omega)
        inst.proc(PVC, "setsmooth")(smooth)
        inst.proc(PVC, "setprecisioncuda")(bool(fp32c))
        p, _, q = new_grid(inst, level)
        _init(inst, "strat", p, q)
        s0 = state(p, q)
        inst.proc(PVC, "initializempirk4")(p, q, rank, nprocs)
        t = t0
        for _ in range(steps):
            inst.proc(PVC, "stratosphererk4")(p, q, t, dt, rank, nprocs)
            t = t + dt
        inst.proc(PVC, "finalizempirk4")()
        return s0, state(p, q)

    res = _ranks(nprocs, body, shim_runner(), {"__cdll__": lib})
    s0, s1 = res[0]
    return dict(initial=s0, final=s1, ranks=[dict(final=r[1]) for r in res])


# ----------------------------------------------------------------------------- the driver
def read_namelist(path) -> dict:
    """The groups of a namelist file (&group key = value ... /) as {group: {key: value}}: integers,
    reals (d exponents too), logicals and quoted strings; text outside a group is ignored."""
    groups, cur = {}, None
    with open(path, encoding="latin-1") as f:
        for raw in f:
            line = raw.split("!")[0].strip()
            if not line:
                continue
            if line.startswith("&"):
                cur = groups.setdefault(line[1:].split()[0].lower(), {})
                continue
            if line.startswith("/"):
                cur = None
                continue
            if cur is None or "=" not in line:
                continue
            for item in line.split(","):
                if "=" not in item:
                    continue
                k, v = (t.strip() for t in item.split("=", 1))
                if v[:1] in "'\"":
                    val = v.strip("'\"")
                elif v.lower() in (".true.", "t", ".false.", "f"):
                    val = v.lower() in (".true.", "t")
                else:
                    try:
                        val = int(v)
                    except ValueError:
                        val = float(v.lower().replace("d", "e"))
                cur[k.lower()] = val
    return groups



def run_driver(nprocs, namelist, cuda=False, lib_path=None, fp32c=False, which="rh4") -> dict:
    """A driver program of the reference on nprocs thread ranks: RHWavePanelsMPI.f90 ("rh4") or
    StratospherePanels.f90 ("strat"), its namelist groups (gridinit, time, fileio) given as dicts,
    with its own PanelVelocityParallelModule (cuda False) or with its `use` line switched to the
    drop-in module and the library at lib_path (cuda True). Returns what rank 0 writes to the
    data file as an array (per step; rh4: totalKE, enstrophy, relVort l1, l2, linf error against
    the steady wave; strat: totalKE, enstrophy), and everything every rank wrote."""
    prog = driver_runner(bool(cuda), which)
    DRV = DRIVERS[which][1]
    lib = _lib(lib_path) if cuda else None
    written = [[] for _ in range(nprocs)]

    def host(rank):
        h = {"__namelist__": {k.lower(): {n.lower(): v for n, v in g.items()} for k, g in namelist.items()},
             "__write__": lambda unit, vals: written[rank].append((int(unit), list(vals)))}
        if lib is not None:
            h["__cdll__"] = lib
        return h

    def body(inst, rank):
        if cuda:
            inst.proc(PVC, "setprecisioncuda")(bool(fp32c))
        inst.proc(DRV, "main")()
        return None

    _ranks(nprocs, body, prog, host)
    data_unit = 13  # writeUnit of the driver
    rows = [[float(v) for v in vals] for unit, vals in written[0]
            if unit == data_unit and vals and not isinstance(vals[0], str)]
    return dict(rows=np.array(rows), written=written)
