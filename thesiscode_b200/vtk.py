"""Legacy-VTK polydata output of a panel grid (vtkOutputUnif,
ParticlesEdgesPanels2.f90:2116-2237).

The file is the reference's ASCII layout, so ParaView/VTK readers and the
reference's post-processing scripts read both alike: header, POINTS (all
particles, F24.18), POLYGONS (one cell per leaf panel, 0-based vertex
indices, I8), POINT_DATA (particle tracers, relVort, absVort) and CELL_DATA
(leaf-panel tracers, relVortPanel, absVortPanel), one value per line in
F24.18. Writing the file needs no graphics library.
"""
from __future__ import annotations

import io
from pathlib import Path

import numpy as np

from .grid import Panels, Particles


def _f24_18(v: float) -> str:
    """Fortran F24.18: 18 decimals right-justified in 24 columns, asterisks when it does not fit."""
    s = f"{v:24.18f}"
    return "*" * 24 if len(s) > 24 else s


def _i8(k: int) -> str:
    s = f"{int(k):8d}"
    return "*" * 8 if len(s) > 8 else s


def _column(out: io.StringIO, values) -> None:
    for v in np.asarray(values, dtype=np.float64).ravel():
        out.write(_f24_18(float(v)) + "\n")


def vtk_text(particles: Particles, panels: Panels) -> str:
    """The vtkOutputUnif file contents for a triangular or quadrilateral panel grid."""
    leaves = ~np.asarray(panels.hasChildren, dtype=bool)
    n_active = int(np.count_nonzero(leaves))
    n_points = particles.x.shape[0]
    verts = np.asarray(panels.vertices)[leaves]
    kind = verts.shape[1]
    if kind not in (3, 4):
        raise ValueError("vtk_text writes triangular or quadrilateral panels")
    n_tracers = particles.tracer.shape[1] if particles.tracer is not None and particles.tracer.ndim == 2 else 0
    out = io.StringIO()
    out.write("# vtk DataFile Version 2.0\n")
    out.write("Sphere Grid : " + _i8(n_active) + " panels.\n")
    out.write("ASCII\n")
    out.write("DATASET POLYDATA\n")
    out.write("POINTS " + _i8(n_points) + "   double\n")
    for p in particles.x:
        out.write(_f24_18(p[0]) + _f24_18(p[1]) + _f24_18(p[2]) + "\n")
    out.write("POLYGONS" + _i8(n_active) + _i8((kind + 1) * n_active) + "\n")
    # panel vertices are 0-based particle indices here (the reference subtracts 1 from its 1-based ones)
    for row in verts:
        out.write(_i8(kind) + "".join(_i8(v) for v in row) + "\n")
    out.write("POINT_DATA   " + _i8(n_points) + "\n")
    for k in range(n_tracers):
        out.write(f" SCALARS  Tracer{k + 1}  double 1\n")
        out.write("LOOKUP_TABLE default\n")
        _column(out, particles.tracer[:, k])
    out.write("SCALARS   relVort  double 1\n")
    out.write("LOOKUP_TABLE default\n")
    _column(out, particles.relVort)
    out.write("SCALARS   absVort  double 1\n")
    out.write("LOOKUP_TABLE default\n")
    _column(out, particles.absVort)
    out.write("CELL_DATA   " + _i8(n_active) + "\n")
    n_panel_tracers = panels.tracer.shape[1] if panels.tracer is not None and panels.tracer.ndim == 2 else 0
    for k in range(min(n_tracers, n_panel_tracers)):
        out.write(f"SCALARS TracerPanel{k + 1} double 1\n")
        out.write("LOOKUP_TABLE default\n")
        _column(out, panels.tracer[leaves, k])
    out.write("SCALARS  relVortPanel  double 1\n")
    out.write("LOOKUP_TABLE default\n")
    _column(out, np.asarray(panels.relVort)[leaves])
    out.write("SCALARS  absVortPanel  double 1\n")
    out.write("LOOKUP_TABLE default\n")
    _column(out, np.asarray(panels.absVort)[leaves])
    return out.getvalue()


def vtk_output_unif(particles: Particles, panels: Panels, filename: str | Path) -> None:
    """vtkOutputUnif: write the grid and its vorticity/tracer fields as legacy VTK polydata."""
    Path(filename).write_text(vtk_text(particles, panels))


def read_vtk_polydata(filename: str | Path) -> dict:
    """Minimal reader of the files vtk_output_unif writes (points, polygons, named scalars)."""
    lines = Path(filename).read_text().splitlines()
    out: dict = {"point_data": {}, "cell_data": {}}
    i = 4
    n_points = int(lines[i].split()[1])
    out["points"] = np.array([[float(lines[i + 1 + j][24 * c:24 * (c + 1)]) for c in range(3)]
                              for j in range(n_points)])
    i += 1 + n_points
    _, n_cells, _ = lines[i].split()
    n_cells = int(n_cells)
    out["polygons"] = np.array([[int(v) for v in lines[i + 1 + j].split()[1:]] for j in range(n_cells)])
    i += 1 + n_cells
    section = None
    while i < len(lines):
        words = lines[i].split()
        if words[0] == "POINT_DATA":
            section, count = "point_data", int(words[1])
            i += 1
        elif words[0] == "CELL_DATA":
            section, count = "cell_data", int(words[1])
            i += 1
        elif words[0] == "SCALARS":
            name = words[1]
            vals = np.array([float(v) for v in lines[i + 2:i + 2 + count]])
            out[section][name] = vals
            i += 2 + count
        else:
            i += 1
    return out
