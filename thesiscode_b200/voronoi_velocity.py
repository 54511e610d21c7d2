"""Host mirror of VoronoiVelocityParallelModule (VoronoiVelocityParallel.f90).

`VorPanels` holds the SoA generator arrays of type(VorPanels)
(VoronoiPanels.f90:25-58) that the velocity path reads; `BVEVelocity`
(:487-515) and `BVERK4` (:304-478) run on the GPU through the C ABI. The
Delaunay/Voronoi rebuild that follows each reference step (:480-482, STRIPACK
on the host) is the caller's.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _native as N
from .panel_velocity import Context


@dataclass
class VorPanels:
    x: np.ndarray        # (N_Max,)
    y: np.ndarray
    z: np.ndarray
    relVort: np.ndarray
    absVort: np.ndarray
    area: np.ndarray
    N: int               # generators in use (1..N); N_Max = len(x)

    @property
    def N_Max(self) -> int:
        return self.x.shape[0]


def BVEVelocity(ctx: Context, x, y, z, vort, area, indexStart: int, indexEnd: int, dy=None, dz=None):
    """One SoA sum; 0-based half-open [indexStart, indexEnd). Returns (dx, dy, dz, dVort) with the
    reference's semantics (dy, dz accumulate into the caller's values; see the C header)."""
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z, vort, area)]
    n = arrs[0].shape[0]
    dx = np.zeros(n)
    dy = np.zeros(n) if dy is None else np.array(dy, dtype=np.float64)
    dz = np.zeros(n) if dz is None else np.array(dz, dtype=np.float64)
    dv = np.zeros(n)
    N.call("tc_bs_velocity_soa", ctx.handle, *[N.dptr(a) for a in arrs], n, int(indexStart), int(indexEnd),
           N.dptr(dx), N.dptr(dy), N.dptr(dz), N.dptr(dv))
    return dx, dy, dz, dv


def BVERK4(ctx: Context, aPanels: VorPanels, dt: float, nsteps: int = 1):
    """Voronoi BVERK4 on the N used generators (updated in place); returns (totalKE per step,
    kineticEnergy). The caller rebuilds the Delaunay/Voronoi structure afterwards."""
    n = aPanels.N
    x, y, z = (np.ascontiguousarray(a[:n]) for a in (aPanels.x, aPanels.y, aPanels.z))
    zeta = np.ascontiguousarray(aPanels.relVort[:n])
    area = np.ascontiguousarray(aPanels.area[:n])
    tke = np.zeros(max(nsteps, 1))
    ke = np.zeros(n)
    N.call("tc_rk4_soa_step", ctx.handle, N.dptr(x), N.dptr(y), N.dptr(z), N.dptr(zeta), N.dptr(area), n,
           float(dt), int(nsteps), N.dptr(tke), N.dptr(ke))
    aPanels.x[:n], aPanels.y[:n], aPanels.z[:n], aPanels.relVort[:n] = x, y, z, zeta
    return tke[:nsteps], ke
