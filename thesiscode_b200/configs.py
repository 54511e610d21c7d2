"""The benchmark workloads as input arrays (synthetic, seeded, FP64).

Each workload is an icosahedral grid with analytic vorticity at the leaf
panel centres (active panels = sources and targets) and the panel vertices
(passive particles = targets). "Config mode" evaluates one delta at all
targets and has no divided-panel targets; "parity mode" reproduces the
reference's three target classes (active delta 0, vertices delta 0, divided
panels delta = smooth = 0.05; PanelVelocityParallel.f90:27, :1318-1410).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import ics
from .grid import gather_panels, new_icos_grid


@dataclass
class Workload:
    name: str
    level: int
    xA: np.ndarray          # (nA, 3) active panel centres
    zetaA: np.ndarray       # (nA,) relative vorticity
    areaA: np.ndarray       # (nA,)
    xV: np.ndarray          # (nV, 3) particles (vertices)
    xQ: np.ndarray          # (nQ, 3) divided panels (empty in config mode)
    omega: float
    deltas: tuple           # (active, vertex, passive)
    dt: float
    steps: int
    meta: dict = field(default_factory=dict)

    @property
    def nA(self):
        return self.xA.shape[0]

    @property
    def nV(self):
        return self.xV.shape[0]

    @property
    def nQ(self):
        return self.xQ.shape[0]

    def interactions_per_step(self) -> int:
        """Pairs evaluated per RK4 step: 4 stages x (nA(nA-1) + (nV + nQ) nA)."""
        nA, nV, nQ = self.nA, self.nV, self.nQ
        return 4 * (nA * (nA - 1) + (nV + nQ) * nA)

    def copy(self) -> "Workload":
        return Workload(self.name, self.level, self.xA.copy(), self.zetaA.copy(), self.areaA.copy(),
                        self.xV.copy(), self.xQ.copy(), self.omega, tuple(self.deltas), self.dt,
                        self.steps, dict(self.meta))


def _grid(level, grid_source=None):
    """(particle positions, active panel centres, their areas, divided panel centres) of the
    icosahedral grid of `level`: from the library's generator, or from `grid_source(level)`
    (a callable returning the same four arrays, e.g. a CPU restatement of the generator)."""
    if grid_source is not None:
        return tuple(np.ascontiguousarray(a, dtype=np.float64) for a in grid_source(level))
    parts, pans = new_icos_grid(level)
    _, xA, _, aA, xQ = gather_panels(pans)
    return parts.x.copy(), xA, aA, xQ


def rh4(level=4, delta=0.0, dt=0.01, steps=10, Omega=2.0 * np.pi, parity=False,
        grid_source=None) -> Workload:
    """Rossby-Haurwitz wave 4 (config 1 at level 4, config 5 at level 8 with delta 0.005)."""
    xV, xA, aA, xQ = _grid(level, grid_source)
    f = ics.rh4_reference if parity else (lambda x: ics.rh4_config(x, Omega))
    zA = f(xA)
    deltas = (0.0, 0.0, 0.05) if parity else (delta, delta, delta)
    xQ = xQ if parity else np.zeros((0, 3))
    return Workload(f"rh4_l{level}", level, xA, zA, aA, xV, xQ, Omega, deltas, dt, steps,
                    dict(ic="rh4_reference" if parity else "rh4 (omega=K=Omega/14)"))


def gaussian(level=7, delta=0.01, dt=0.01, steps=1, Omega=2.0 * np.pi, parity=False,
             grid_source=None) -> Workload:
    """Gaussian vortex exp(-16|x-x0|^2) at (22.5N, 0E) minus its area mean (config 2 at level 7)."""
    xV, xA, aA, xQ = _grid(level, grid_source)
    g = ics.gaussian_config(xA)
    zA = g - ics.remove_area_mean(g, aA)
    deltas = (0.0, 0.0, 0.05) if parity else (delta, delta, delta)
    xQ = xQ if parity else np.zeros((0, 3))
    return Workload(f"gaussian_l{level}", level, xA, zA, aA, xV, xQ, Omega, deltas, dt,
                    steps, dict(ic="exp(-16|x-x0|^2) - mean, x0=(22.5N,0E)"))


def jet(level=6, delta=0.02, dt=0.005, steps=20, Omega=2.0 * np.pi, U=1.0, noise=1e-2, seed=3,
        grid_source=None) -> Workload:
    """Zonal jet -U sech^2 tanh /0.1 (U = 1) + 1e-2 N(0,1) (seed 3) (config 3 at level 6)."""
    xV, xA, aA, xQ = _grid(level, grid_source)
    rng = np.random.default_rng(seed)
    zA = ics.jet_config(xA, U=U) + noise * rng.standard_normal(xA.shape[0])
    return Workload(f"jet_l{level}", level, xA, zA, aA, xV, np.zeros((0, 3)), Omega,
                    (delta, delta, delta), dt, steps, dict(ic="jet U=1 + 1e-2 N(0,1) seed 3"))


def solid_body(level=3, rotation_rate=2.0 * np.pi, dt=0.01, steps=1) -> Workload:
    """Solid-body rotation known answer (solidBody.f90, SolidBody.namelist): zeta = 2 w z, Omega = 0."""
    xV, xA, aA, xQ = _grid(level)
    zA = ics.solid_body(xA, rotation_rate)
    return Workload(f"solid_body_l{level}", level, xA, zA, aA, xV, np.zeros((0, 3)), 0.0,
                    (0.0, 0.0, 0.0), dt, steps, dict(rotation_rate=rotation_rate))


def stratosphere(level=4, dt=0.01, steps=1, t0=5.0, Omega=2.0 * np.pi, parity=True) -> Workload:
    """Forced stratosphere model (InitStratosphere, TracerAndVorticityDistributions.f90:793-824;
    StratosphereRK4, PanelVelocityParallel.f90:661-919): relVort = StratosphereRelVortX - gaussConst,
    absVort = relVort + 2 Omega z at panels and vertices; meta holds absVortA, absVortV and the start
    time t0 (the Juckes forcing is fully on for 4 <= t < 11)."""
    xV, xA, aA, xQ = _grid(level)
    g = ics.stratosphere_rel_vort(xA)
    gc = ics.remove_area_mean(g, aA)
    zA = g - gc
    absA = zA + 2.0 * Omega * xA[:, 2]
    absV = ics.stratosphere_rel_vort(xV) - gc + 2.0 * Omega * xV[:, 2]
    deltas = (0.0, 0.0, 0.05)
    xQ = xQ if parity else np.zeros((0, 3))
    return Workload(f"stratosphere_l{level}", level, xA, zA, aA, xV, xQ, Omega, deltas, dt, steps,
                    dict(ic="StratosphereRelVortX - gaussConst", absVortA=absA, absVortV=absV, t0=t0))


def batched_gaussians(count=64, seed=4, levels=(3, 4, 5, 6), dt=0.01, steps=10,
                      Omega=2.0 * np.pi, delta=0.0, grid_source=None) -> list[Workload]:
    """Config 4: independent Gaussian vortices, level ~ U{3..6}, centre uniform on the sphere,
    beta ~ U[4, 20], zeta = exp(-beta^2 |x - x0|^2) minus its area mean (seed 4)."""
    rng = np.random.default_rng(seed)
    grids = {}
    out = []
    for k in range(count):
        level = int(rng.choice(levels))
        v = rng.standard_normal(3)
        x0 = v / np.linalg.norm(v)
        beta = rng.uniform(4.0, 20.0)
        if level not in grids:
            grids[level] = _grid(level, grid_source)
        xV, xA, aA, xQ = grids[level]
        d = xA - x0
        g = np.exp(-beta * beta * np.einsum("ij,ij->i", d, d))
        zA = g - ics.remove_area_mean(g, aA)
        out.append(Workload(f"batch{k}_l{level}", level, xA.copy(), zA, aA.copy(), xV.copy(),
                            np.zeros((0, 3)), Omega, (delta, delta, delta), dt, steps,
                            dict(beta=beta, x0=x0.tolist())))
    return out
