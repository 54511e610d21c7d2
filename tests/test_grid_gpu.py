"""The icosahedral grid generated on the GPU (tc_icos_grid_device) against the host generator
(tc_icos_grid, which restates InitIcosTriGrid / DivideTriPanel / TriPanelArea,
ParticlesEdgesPanels2.f90:419-1090, :1727-1802): the same numbering, bitwise the same positions
and centres, areas within a few ulps."""
import numpy as np
import pytest

from thesiscode_b200 import grid
from thesiscode_b200.panel_velocity import Context


@pytest.mark.gpu
@pytest.mark.parametrize("level", [0, 1, 2, 5, 8])
def test_device_grid_equals_host_grid(gpu, level):
    parts, pans = grid.new_icos_grid(level)
    ctx = Context(0, "fp64")
    try:
        d = {k: v.cpu().numpy() for k, v in grid.new_icos_grid_device(ctx, level).items()}
    finally:
        ctx.close()
    assert np.array_equal(d["particles_x"], parts.x)
    assert np.array_equal(d["particles_x0"], parts.x0)
    assert np.array_equal(d["panels_x"], pans.x)
    assert np.array_equal(d["panels_x0"], pans.x0)
    assert np.array_equal(d["panels_has_children"].astype(bool), pans.hasChildren)
    assert np.array_equal(d["panels_vertices"], pans.vertices)
    assert np.array_equal(d["panels_nest"], pans.nest)
    assert np.array_equal(d["panels_children"], pans.children)
    # areas: CUDA's atan2 / tan against the host's, a few ulps of each panel's area
    assert np.abs(d["panels_area"] - pans.area).max() <= 1e-14 * pans.area.max()
    leaves = ~pans.hasChildren
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
