"""The icosahedral grid generated on the GPU (tc_icos_grid_device) against the oracle's
restatement of InitIcosTriGrid / DivideTriPanel / TriPanelArea (oracle/icos_oracle.c,
ParticlesEdgesPanels2.f90:419-1090, :1727-1802), which the host generator tc_icos_grid equals bit
for bit: the same numbering, bitwise the same positions and centres, areas within a few ulps."""
import numpy as np
import pytest

from thesiscode_b200 import grid
from thesiscode_b200.panel_velocity import Context


@pytest.mark.gpu
@pytest.mark.parametrize("level", [0, 1, 2, 5, 8])
def test_device_grid_equals_oracle_grid(gpu, level):
    from oracle import oracle as O

    ref = O.icos_grid(level)
    ctx = Context(0, "fp64")
    try:
        d = {k: v.cpu().numpy() for k, v in grid.new_icos_grid_device(ctx, level).items()}
    finally:
        ctx.close()
    for k in ("particles_x", "particles_x0", "panels_x", "panels_x0", "panels_has_children",
              "panels_vertices", "panels_nest", "panels_children"):
        assert np.array_equal(d[k], ref[k]), k
    # areas: CUDA's atan2 / tan against the host libm's, a few ulps of each panel's area
    assert np.abs(d["panels_area"] - ref["panels_area"]).max() <= 1e-14 * ref["panels_area"].max()
    leaves = ref["panels_has_children"] == 0
    assert abs(d["panels_area"][leaves].sum() - 4 * np.pi) <= 1e-12


@pytest.mark.gpu
def test_device_grid_rejects_bad_level(gpu):
    from thesiscode_b200 import _native as N

    ctx = Context(0, "fp64")
    try:
        with pytest.raises(N.TcError) as e:
            grid.new_icos_grid_device(ctx, 12)
        assert e.value.status == N.TC_ERR_ARG
    finally:
        ctx.close()


@pytest.mark.gpu
def test_device_grid_equals_the_reference_grid(gpu):
    """The same at level 3 against the reference's own NewGrid, run from its Fortran source by
    oracle/f90 (tests/golden/ref_grid_l3.npz)."""
    from pathlib import Path

    ref = np.load(Path(__file__).resolve().parent / "golden" / "ref_grid_l3.npz")
    ctx = Context(0, "fp64")
    try:
        d = {k: v.cpu().numpy() for k, v in grid.new_icos_grid_device(ctx, 3).items()}
    finally:
        ctx.close()
    for k in ("particles_x", "particles_x0", "panels_x", "panels_x0", "panels_has_children",
              "panels_vertices", "panels_nest", "panels_children"):
        assert np.array_equal(d[k], ref[k]), k
    assert np.abs(d["panels_area"] - ref["panels_area"]).max() <= 1e-14 * ref["panels_area"].max()
