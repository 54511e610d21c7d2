"""ctypes wrapper of the CPU FP64 oracle (oracle/bve_oracle.c, oracle/strat_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by the entry module's smoke() to
verify one GPU step, and by bench.py's CPU-baseline leg. The product never imports
it. Parity status: pinned against the reference's own code. The reference is
Fortran and no Fortran compiler is available to build it, so its source runs
through oracle/f90 (a translator of the Fortran 90 subset its modules use,
strict IEEE double arithmetic); this oracle equals those runs bit for bit
(tests/test_reference_source.py), and the reference drivers' known answers
hold for it (tests/test_oracle.py).
"""
from __future__ import annotations

import ctypes
import subprocess
from ctypes import POINTER, c_double, c_int
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"

dp = POINTER(c_double)
ip = POINTER(c_int)

_lib = None
_fast: dict = {}

# x86-64 ISA levels of the timing builds and the /proc/cpuinfo flags each needs
# (the psABI's x86-64-v3 and v4 feature lists).
_LEVELS = (
    ("v4", {"avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl"}),
    ("v3", {"avx", "avx2", "bmi1", "bmi2", "f16c", "fma", "abm", "movbe", "xsave"}),
)


def build() -> Path:
    """Compile the oracle with its Makefile: the strict parity build (gcc -O2
    -ffp-contract=off) and the timing builds."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def host_isa_level() -> str:
    """The highest x86-64 level (v4, v3, else sse2) whose features the host CPU reports."""
    try:
        with open("/proc/cpuinfo") as f:
            flags = next((set(line.split(":", 1)[1].split()) for line in f if line.startswith("flags")),
                         set())
    except OSError:
        flags = set()
    for name, need in _LEVELS:
        if need <= flags:
            return name
    return "sse2"


def fast_lib(level: str | None = None):
    """(handle, ISA level) of a timing build: the same loops compiled like the reference's
    ifort -O2 (reassociation, reciprocal division, contraction, vectorized), for `level` (default:
    the host's highest). A level above the host's is refused: its code would not run here."""
    order = ["sse2", "v3", "v4"]
    host = host_isa_level()
    level = level or host
    if order.index(level) > order.index(host):
        raise ValueError(f"x86-64-{level} build needs CPU features this host lacks (host: {host})")
    if level not in _fast:
        path = HERE / "_build" / f"liboracle_fast_{level}.so"
        if not path.exists():
            build()
        h = ctypes.CDLL(str(path))
        h.or_rows.argtypes = [c_int, ip, c_int, dp, dp, dp, dp, c_int, c_double, dp, c_int]
        _fast[level] = h
    return _fast[level], level


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        h = ctypes.CDLL(str(LIB))
        h.or_active_rhs.argtypes = [dp, dp, dp, dp, dp, c_int, c_int, c_int, c_double, c_double]
        h.or_passive_rhs.argtypes = [dp, dp, c_int, dp, dp, dp, c_int, c_int, c_int]
        h.or_smooth_velocity.argtypes = [dp, dp, c_int, dp, dp, dp, c_int, c_int, c_int, c_double]
        h.or_voronoi_velocity.argtypes = [dp, dp, dp, dp, dp, dp, dp, dp, dp, c_int, c_int, c_int,
                                          c_double]
        h.or_rows.argtypes = [c_int, ip, c_int, dp, dp, dp, dp, c_int, c_double, dp, c_int]
        h.or_load_balance.argtypes = [c_int, c_int, ip, ip]
        h.or_bve_rk4.argtypes = [dp, c_int, dp, dp, dp, c_int, dp, c_int, c_double, c_double,
                                 c_double, c_double, c_double, dp, dp, dp, c_int]
        h.or_bve_rk4.restype = c_double
        h.or_bve_stage.argtypes = [dp, dp, dp, c_int, dp, c_int, dp, c_int, c_double, c_double,
                                   c_double, c_double, c_int, c_int, c_int, c_int, c_int, c_int,
                                   dp, dp, dp, dp, c_int]
        h.or_juckes_forcing.argtypes = [dp, c_double]
        h.or_juckes_forcing.restype = c_double
        h.or_juckes_a.argtypes = [c_double]
        h.or_juckes_a.restype = c_double
        h.or_strat_rk4.argtypes = [dp, c_int, dp, dp, dp, dp, c_int, dp, c_int, dp, dp, c_double,
                                   c_double, c_double, c_double, c_double, c_double, dp, c_int]
        h.or_strat_rk4.restype = c_double
        h.or_icos_sizes.argtypes = [c_int, ip, ip, ip, ip]
        h.or_icos_grid.argtypes = [c_int, dp, dp, dp, dp, dp, ip, ip, ip, ip]
        h.or_gather_maps.argtypes = [c_int, ip, ip, c_int, ip, c_int]
        _lib = h
    return _lib


def _d(a):
    return None if a is None else a.ctypes.data_as(dp)


def _c(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def active_rhs(x, vort, area, i0=0, i1=None, omega=2 * np.pi, delta=0.0):
    """BVEActiveRHS -> (dX (n,3), dVort (n,))."""
    x, vort, area = _c(x), _c(vort), _c(area)
    n = x.shape[0]
    i1 = n if i1 is None else i1
    dX = np.zeros((n, 3))
    dV = np.zeros(n)
    lib().or_active_rhs(_d(dX), _d(dV), _d(x), _d(vort), _d(area), n, i0, i1, omega, delta)
    return dX, dV


def passive_rhs(X, x, vort, area, i0=0, i1=None):
    """BVEPassiveRHS -> dX (m,3)."""
    X, x, vort, area = _c(X), _c(x), _c(vort), _c(area)
    m = X.shape[0]
    i1 = m if i1 is None else i1
    dX = np.zeros((m, 3))
    lib().or_passive_rhs(_d(dX), _d(X), m, _d(x), _d(vort), _d(area), x.shape[0], i0, i1)
    return dX


def smooth_velocity(X, x, vort, area, smooth=0.05, i0=0, i1=None):
    """BVESmoothVelocity -> dX (m,3)."""
    X, x, vort, area = _c(X), _c(x), _c(vort), _c(area)
    m = X.shape[0]
    i1 = m if i1 is None else i1
    dX = np.zeros((m, 3))
    lib().or_smooth_velocity(_d(dX), _d(X), m, _d(x), _d(vort), _d(area), x.shape[0], i0, i1, smooth)
    return dX


def voronoi_velocity(x, y, z, vort, area, i0=0, i1=None, omega=2 * np.pi, dy=None, dz=None):
    """BVEVelocity (Voronoi SoA) -> (dx, dy, dz, dVort)."""
    x, y, z, vort, area = map(_c, (x, y, z, vort, area))
    n = x.shape[0]
    i1 = n if i1 is None else i1
    dx = np.zeros(n)
    dy = np.zeros(n) if dy is None else _c(dy).copy()
    dz = np.zeros(n) if dz is None else _c(dz).copy()
    dV = np.zeros(n)
    lib().or_voronoi_velocity(_d(dx), _d(dy), _d(dz), _d(dV), _d(x), _d(y), _d(z), _d(vort), _d(area),
                              n, i0, i1, omega)
    return dx, dy, dz, dV


def rows(cls, row_idx, X, x, vort, area, delta=0.0, nthreads=1, fast=False):
    """Sums for a list of target rows (cls 0 active / 1 vertex / 2 passive) -> (r,3).
    fast=True (or an ISA level name) runs a timing build (fast_lib) instead of the strict
    parity build."""
    row_idx = np.ascontiguousarray(row_idx, dtype=np.int32)
    x, vort, area = _c(x), _c(vort), _c(area)
    Xc = None if X is None else _c(X)
    out = np.zeros((row_idx.shape[0], 3))
    h = fast_lib(fast if isinstance(fast, str) else None)[0] if fast else lib()
    h.or_rows(int(cls), row_idx.ctypes.data_as(ip), row_idx.shape[0], _d(Xc), _d(x), _d(vort),
              _d(area), x.shape[0], delta, _d(out), nthreads)
    return out


def load_balance(n, p):
    s = np.zeros(p, np.int32)
    e = np.zeros(p, np.int32)
    lib().or_load_balance(n, p, s.ctypes.data_as(ip), e.ctypes.data_as(ip))
    return s, e


def bve_rk4(xV, xA, zetaA, areaA, xQ, dt, omega=2 * np.pi, deltas=(0.0, 0.0, 0.05),
            absVortV=None, nthreads=1):
    """One BVERK4 step on copies; returns (xV, xA, zetaA, xQ, totalKE, kineticEnergy, relVortV)."""
    xV, xA, zetaA, areaA, xQ = (_c(a).copy() for a in (xV, xA, zetaA, areaA, xQ))
    ke = np.zeros(xA.shape[0])
    rel = None
    absV = None
    if absVortV is not None:
        absV = _c(absVortV)
        rel = np.zeros(xV.shape[0])
    tke = lib().or_bve_rk4(_d(xV), xV.shape[0], _d(xA), _d(zetaA), _d(areaA), xA.shape[0], _d(xQ),
                           xQ.shape[0], dt, omega, deltas[0], deltas[1], deltas[2], _d(absV), _d(rel),
                           _d(ke), nthreads)
    return xV, xA, zetaA, xQ, tke, ke, rel


def bve_stage(xA, zetaA, areaA, xV, xQ, omega, deltas, ranges, nthreads=1):
    """One stage's three sums over the given ranges (a0,a1,v0,v1,q0,q1)."""
    xA, zetaA, areaA, xV, xQ = map(_c, (xA, zetaA, areaA, xV, xQ))
    nA, nV, nQ = xA.shape[0], xV.shape[0], xQ.shape[0]
    dXA = np.zeros((nA, 3))
    dVA = np.zeros(nA)
    dXV = np.zeros((nV, 3))
    dXQ = np.zeros((nQ, 3))
    lib().or_bve_stage(_d(xA), _d(zetaA), _d(areaA), nA, _d(xV), nV, _d(xQ), nQ, omega, deltas[0],
                       deltas[1], deltas[2], *[int(r) for r in ranges], _d(dXA), _d(dVA), _d(dXV),
                       _d(dXQ), nthreads)
    return dXA, dVA, dXV, dXQ


def juckes_forcing(x, t):
    """Juckes forcing F(x, t) at each row of x (n,3)."""
    x = _c(np.atleast_2d(x))
    return np.array([lib().or_juckes_forcing(_d(np.ascontiguousarray(r)), float(t)) for r in x])


def strat_rk4(xV, xA, absVortA, areaA, xQ, t, dt, omega=2 * np.pi, deltas=(0.0, 0.0, 0.05),
              absVortV=None, nthreads=1):
    """One StratosphereRK4 step from time t on copies; returns
    (xV, xA, relVortA, xQ, totalKE, kineticEnergy, relVortV)."""
    xV, xA, absA, areaA, xQ = (_c(a).copy() for a in (xV, xA, absVortA, areaA, xQ))
    nA = xA.shape[0]
    ke = np.zeros(nA)
    relA = np.zeros(nA)
    relV = absV = None
    if absVortV is not None:
        absV = _c(absVortV)
        relV = np.zeros(xV.shape[0])
    tke = lib().or_strat_rk4(_d(xV), xV.shape[0], _d(xA), _d(absA), _d(relA), _d(areaA), nA, _d(xQ),
                             xQ.shape[0], _d(absV), _d(relV), t, dt, omega, deltas[0], deltas[1],
                             deltas[2], _d(ke), nthreads)
    return xV, xA, relA, xQ, tke, ke, relV


def icos_sizes(level):
    """(particles, edges, panels, active panels) of icosahedral level `level` (PanelMax,
    ParticleMax, EdgeMax: ParticlesEdgesPanels2.f90:2614-2662)."""
    v = [c_int() for _ in range(4)]
    if lib().or_icos_sizes(int(level), *[ctypes.byref(x) for x in v]) != 0:
        raise ValueError(f"icosahedral level {level} outside [0, 11]")
    return tuple(x.value for x in v)


def icos_grid(level):
    """The oracle's icosahedral grid (InitIcosTriGrid, ParticlesEdgesPanels2.f90:419-645): a dict
    of particle positions / Lagrangian coordinates and panel centres, Lagrangian centres, areas,
    hasChildren, vertices, nest and children, indices 0-based (-1 = none)."""
    npart, _, npan, _ = icos_sizes(level)
    g = dict(particles_x=np.zeros((npart, 3)), particles_x0=np.zeros((npart, 3)),
             panels_x=np.zeros((npan, 3)), panels_x0=np.zeros((npan, 3)), panels_area=np.zeros(npan),
             panels_has_children=np.zeros(npan, np.int32), panels_vertices=np.zeros((npan, 3), np.int32),
             panels_nest=np.zeros(npan, np.int32), panels_children=np.zeros((npan, 4), np.int32))
    rc = lib().or_icos_grid(int(level), *[_d(g[k]) for k in ("particles_x", "particles_x0", "panels_x",
                                                           "panels_x0", "panels_area")],
                            *[g[k].ctypes.data_as(ip) for k in ("panels_has_children", "panels_vertices",
                                                                 "panels_nest", "panels_children")])
    if rc != 0:
        raise RuntimeError(f"or_icos_grid({level}) failed")
    return g


def gather_maps(has_children):
    """GatherPanels maps (ParticlesEdgesPanels2.f90:1556-1619): (active, passive) panel indices."""
    hc = np.ascontiguousarray(has_children, dtype=np.int32)
    n = hc.shape[0]
    nq = int(np.count_nonzero(hc))
    am, pm = np.zeros(n - nq, np.int32), np.zeros(nq, np.int32)
    if lib().or_gather_maps(n, hc.ctypes.data_as(ip), am.ctypes.data_as(ip), n - nq,
                            pm.ctypes.data_as(ip), nq) != 0:
        raise RuntimeError("or_gather_maps: inconsistent counts")
    return am, pm


def gathered_grid(level):
    """Inputs of a workload on the oracle's grid: (particle positions (nV,3), active panel
    centres (nA,3), their areas (nA,), divided panel centres (nQ,3)); the same arrays the product
    builds with its own generator and GatherPanels maps."""
    g = icos_grid(level)
    am, pm = gather_maps(g["panels_has_children"])
    return (g["particles_x"].copy(), np.ascontiguousarray(g["panels_x"][am]),
            np.ascontiguousarray(g["panels_area"][am]), np.ascontiguousarray(g["panels_x"][pm]))
