"""Particles / Panels data model and the icosahedral grid (host side).

Mirrors the reference's derived types (ParticlesEdgesPanels2.f90:45-89)
with numpy arrays. A Fortran ``x(3,N)`` column-major array is stored here as
a C-ordered ``(N, 3)`` float64 array, which is the same memory layout, so
``x`` can be handed to the C ABI (and to a Fortran caller) without copies.
Indices are 0-based.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _native as N


@dataclass
class Particles:
    """type(Particles), ParticlesEdgesPanels2.f90:45-56 (vertices of panels)."""

    x: np.ndarray                      # (N, 3) positions
    x0: np.ndarray                     # (N, 3) Lagrangian coordinates
    absVort: np.ndarray                # (N,)
    relVort: np.ndarray                # (N,)
    tracer: np.ndarray                 # (N, nTracer)

    @property
    def N(self) -> int:
        return self.x.shape[0]


@dataclass
class Panels:
    """type(Panels), ParticlesEdgesPanels2.f90:71-89."""

    x: np.ndarray                      # (N, 3) centres (a divided panel holds its centre child's)
    x0: np.ndarray
    area: np.ndarray                   # (N,) 0 for divided panels
    hasChildren: np.ndarray            # (N,) bool
    vertices: np.ndarray               # (N, 3) particle indices
    nest: np.ndarray                   # (N,)
    children: np.ndarray               # (N, 4), -1 for leaves
    absVort: np.ndarray
    relVort: np.ndarray
    tracer: np.ndarray                 # (N, nTracer)

    @property
    def N(self) -> int:
        return self.x.shape[0]

    @property
    def N_Active(self) -> int:
        return int(np.count_nonzero(~self.hasChildren))


def icos_sizes(level: int) -> dict:
    """PanelMax / ParticleMax / EdgeMax (ParticlesEdgesPanels2.f90:2614-2662)."""
    import ctypes

    vals = [ctypes.c_int() for _ in range(4)]
    N.call("tc_icos_grid_sizes", level, *[ctypes.byref(v) for v in vals])
    return dict(particles=vals[0].value, edges=vals[1].value, panels=vals[2].value,
                active=vals[3].value)


def new_icos_grid(level: int, n_tracer: int = 0) -> tuple[Particles, Panels]:
    """NewGrid(..., TRI_PANEL, initNest=level, AMR=0, ...) (ParticlesEdgesPanels2.f90:362-396)."""
    s = icos_sizes(level)
    npart, npan = s["particles"], s["panels"]
    px = np.zeros((npart, 3))
    px0 = np.zeros((npart, 3))
    cx = np.zeros((npan, 3))
    cx0 = np.zeros((npan, 3))
    area = np.zeros(npan)
    hc = np.zeros(npan, np.int32)
    verts = np.zeros((npan, 3), np.int32)
    nest = np.zeros(npan, np.int32)
    children = np.zeros((npan, 4), np.int32)
    N.call("tc_icos_grid", level, N.dptr(px), N.dptr(px0), N.dptr(cx), N.dptr(cx0), N.dptr(area),
           N.iptr(hc), N.iptr(verts), N.iptr(nest), N.iptr(children))
    parts = Particles(x=px, x0=px0, absVort=np.zeros(npart), relVort=np.zeros(npart),
                      tracer=np.zeros((npart, n_tracer)))
    pans = Panels(x=cx, x0=cx0, area=area, hasChildren=hc.astype(bool), vertices=verts, nest=nest,
                  children=children, absVort=np.zeros(npan), relVort=np.zeros(npan),
                  tracer=np.zeros((npan, n_tracer)))
    return parts, pans


def new_icos_grid_device(ctx, level: int) -> dict:
    """The grid of new_icos_grid generated on the GPU of `ctx` (tc_icos_grid_device): a dict of
    torch CUDA tensors (particles x, x0; panels x, x0, area, hasChildren, vertices, nest,
    children) in the host generator's numbering and shapes."""
    import torch

    from . import _native as N

    s = icos_sizes(level)
    npart, npan = s["particles"], s["panels"]
    dev = torch.device(f"cuda:{ctx.device}")
    f64 = dict(dtype=torch.float64, device=dev)
    i32 = dict(dtype=torch.int32, device=dev)
    out = dict(particles_x=torch.empty((npart, 3), **f64), particles_x0=torch.empty((npart, 3), **f64),
               panels_x=torch.empty((npan, 3), **f64), panels_x0=torch.empty((npan, 3), **f64),
               panels_area=torch.empty(npan, **f64), panels_has_children=torch.empty(npan, **i32),
               panels_vertices=torch.empty((npan, 3), **i32), panels_nest=torch.empty(npan, **i32),
               panels_children=torch.empty((npan, 4), **i32))
    ptr = [ctypes.c_void_p(t.data_ptr()) for t in out.values()]
    N.call("tc_icos_grid_device", ctx.handle, level, *ptr)
    return out


@dataclass
class GatherMaps:
    """activeMap / passiveMap of GatherPanels (ParticlesEdgesPanels2.f90:1556-1619)."""

    active: np.ndarray
    passive: np.ndarray
    extra: dict = field(default_factory=dict)


def gather_maps(panels: Panels) -> GatherMaps:
    """Leaf panels in index order -> active, divided panels -> passive."""
    n = panels.N
    na = panels.N_Active
    hc = np.ascontiguousarray(panels.hasChildren.astype(np.int32))
    am = np.zeros(na, np.int32)
    pm = np.zeros(n - na, np.int32)
    N.call("tc_gather_maps", n, N.iptr(hc), N.iptr(am), na, N.iptr(pm), n - na)
    return GatherMaps(active=am, passive=pm)


def gather_panels(panels: Panels, maps: GatherMaps | None = None):
    """GatherPanels: (maps, xA, relVortA, areaA, xQ) as contiguous copies."""
    maps = maps or gather_maps(panels)
    xA = np.ascontiguousarray(panels.x[maps.active])
    zA = np.ascontiguousarray(panels.relVort[maps.active])
    aA = np.ascontiguousarray(panels.area[maps.active])
    xQ = np.ascontiguousarray(panels.x[maps.passive])
    return maps, xA, zA, aA, xQ


def scatter_panels(panels: Panels, maps: GatherMaps, xA, relVortA, xQ) -> None:
    """ScatterPanels (ParticlesEdgesPanels2.f90:1622-1637)."""
    panels.x[maps.active] = xA
    panels.relVort[maps.active] = relVortA
    panels.x[maps.passive] = xQ
