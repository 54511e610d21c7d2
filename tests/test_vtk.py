"""Legacy-VTK grid output (vtkOutputUnif, ParticlesEdgesPanels2.f90:2116-2237): layout and round trip."""
import numpy as np

from thesiscode_b200 import grid, ics
from thesiscode_b200.vtk import read_vtk_polydata, vtk_output_unif, vtk_text


def make_grid(level=2, n_tracer=2):
    parts, pans = grid.new_icos_grid(level, n_tracer)
    parts.relVort[:] = ics.stratosphere_rel_vort(parts.x)
    parts.absVort[:] = parts.relVort + 4.0 * np.pi * parts.x[:, 2]
    pans.relVort[:] = ics.stratosphere_rel_vort(pans.x)
    pans.absVort[:] = pans.relVort + 4.0 * np.pi * pans.x[:, 2]
    parts.tracer[:, 0] = parts.x[:, 0]
    pans.tracer[:, 1] = pans.area
    return parts, pans


def test_vtk_layout_matches_reference_format():
    parts, pans = make_grid()
    lines = vtk_text(parts, pans).splitlines()
    n_act = pans.N_Active
    assert lines[0] == "# vtk DataFile Version 2.0"
    assert lines[1] == f"Sphere Grid : {n_act:8d} panels."
    assert lines[2:4] == ["ASCII", "DATASET POLYDATA"]
    assert lines[4] == f"POINTS {parts.N:8d}   double"
    assert len(lines[5]) == 72  # 3 x F24.18
    assert lines[5 + parts.N] == f"POLYGONS{n_act:8d}{4 * n_act:8d}"
    assert len(lines[6 + parts.N]) == 32  # I8 count + 3 x I8
    assert f"POINT_DATA   {parts.N:8d}" in lines
    assert " SCALARS  Tracer1  double 1" in lines
    assert f"CELL_DATA   {n_act:8d}" in lines
    assert "SCALARS TracerPanel2 double 1" in lines
    # header + points + polygons + point data (2 tracers, relVort, absVort) + cell data (same)
    expect = 5 + parts.N + 1 + n_act + 1 + 4 * (2 + parts.N) + 1 + 4 * (2 + n_act)
    assert len(lines) == expect


def test_vtk_round_trip(tmp_path):
    parts, pans = make_grid(level=3)
    f = tmp_path / "grid.vtk"
    vtk_output_unif(parts, pans, f)
    d = read_vtk_polydata(f)
    leaves = ~pans.hasChildren
    assert np.abs(d["points"] - parts.x).max() <= 5e-19
    assert np.array_equal(d["polygons"], pans.vertices[leaves])
    assert d["polygons"].min() >= 0 and d["polygons"].max() < parts.N
    assert np.abs(d["point_data"]["relVort"] - parts.relVort).max() <= 5e-18 * 16
    assert np.abs(d["cell_data"]["absVortPanel"] - pans.absVort[leaves]).max() <= 5e-17
    assert np.abs(d["cell_data"]["TracerPanel2"] - pans.area[leaves]).max() <= 5e-19
    assert np.abs(d["point_data"]["Tracer1"] - parts.x[:, 0]).max() <= 5e-19


def test_f24_18_overflow_is_asterisks():
    from thesiscode_b200.vtk import _f24_18
    assert _f24_18(-0.5) == "   -0.500000000000000000"
    assert _f24_18(1e6) == "*" * 24


def test_vtk_text_equals_the_reference_writer():
    """The reference's own vtkOutputUnif (its Fortran source run by oracle/f90: formatted WRITEs
    with FORMAT labels and list-directed lines, collected as text; tests/golden/ref_vtk_l1.npz) and
    vtk_text on the library's grid with the same field values write the same file, byte for byte."""
    from pathlib import Path

    f = np.load(Path(__file__).resolve().parent / "golden" / "ref_vtk_l1.npz")
    parts, pans = grid.new_icos_grid(1, 2)
    parts.relVort[:], parts.absVort[:] = f["particles_relVort"], f["particles_absVort"]
    parts.tracer[:] = f["particles_tracer"]
    pans.relVort[:], pans.absVort[:] = f["panels_relVort"], f["panels_absVort"]
    pans.tracer[:] = f["panels_tracer"]
    assert vtk_text(parts, pans) == str(f["text"])
