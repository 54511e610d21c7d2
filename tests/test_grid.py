"""Icosahedral grid generator (host C++ in the library; no GPU needed):
counts of PanelMax/ParticleMax, total area 4 pi (PrintStats check,
ParticlesEdgesPanels2.f90:2089), unit-sphere centres, quad-tree structure
and the GatherPanels order."""
import numpy as np
import pytest

from thesiscode_b200 import grid


@pytest.fixture(scope="module", autouse=True)
def _built(native_built):
    return native_built


@pytest.mark.parametrize("level", [0, 1, 2, 3, 4, 5])
def test_counts_and_area(level):
    parts, pans = grid.new_icos_grid(level)
    assert parts.N == 2 + 10 * 4 ** level
    assert pans.N == sum(20 * 4 ** j for j in range(level + 1))
    assert pans.N_Active == 20 * 4 ** level
    assert abs(pans.area.sum() - 4 * np.pi) < 1e-12
    assert np.all(pans.area[pans.hasChildren] == 0.0)
    assert np.all(pans.area[~pans.hasChildren] > 0.0)
    np.testing.assert_allclose(np.linalg.norm(pans.x, axis=1), 1.0, atol=1e-15)
    np.testing.assert_allclose(np.linalg.norm(parts.x, axis=1), 1.0, atol=1e-15)


def test_icosahedron_vertices_and_root_panels():
    parts, pans = grid.new_icos_grid(0)
    np.testing.assert_array_equal(parts.x[0], [0, 0, 1])
    np.testing.assert_array_equal(parts.x[11], [0, 0, -1])
    # panel 1 of the reference has vertices [1,2,3] (1-based)
    assert list(pans.vertices[0]) == [0, 1, 2]
    np.testing.assert_allclose(pans.area, 4 * np.pi / 20, rtol=1e-13)


def test_children_numbering_and_parent_position():
    parts, pans = grid.new_icos_grid(2)
    # root panels 0..19 divided first, children appended in order (DivideTriPanel :760-1090)
    for p in range(20):
        assert list(pans.children[p]) == [20 + 4 * p + j for j in range(4)]
        assert pans.nest[pans.children[p, 0]] == 1
    # a divided panel copies its centre child's position when it is divided (:1075-1076);
    # level-1 children are divided later and move to their own centre child's position
    _, p1 = grid.new_icos_grid(1)
    for p in range(20):
        np.testing.assert_array_equal(p1.x[p], p1.x[p1.children[p, 3]])
    for p in range(20, 100):
        np.testing.assert_array_equal(pans.x[p], pans.x[pans.children[p, 3]])
    # shared edge midpoints: every vertex of level 2 is used by 5 or 6 leaf panels
    leaves = pans.vertices[~pans.hasChildren]
    counts = np.bincount(leaves.ravel(), minlength=parts.N)
    assert set(np.unique(counts)) <= {5, 6}
    assert np.count_nonzero(counts == 5) == 12


def test_gather_maps_order():
    parts, pans = grid.new_icos_grid(3)
    maps = grid.gather_maps(pans)
    np.testing.assert_array_equal(maps.active, np.nonzero(~pans.hasChildren)[0])
    np.testing.assert_array_equal(maps.passive, np.nonzero(pans.hasChildren)[0])
    m, xA, zA, aA, xQ = grid.gather_panels(pans, maps)
    x = pans.x.copy()
    grid.scatter_panels(pans, maps, xA + 1.0, zA, xQ)
    np.testing.assert_array_equal(pans.x[maps.active], x[maps.active] + 1.0)


def test_bad_level_is_an_error():
    from thesiscode_b200 import _native as N

    with pytest.raises(N.TcError):
        grid.icos_sizes(12)


_FIELDS = ("particles_x", "particles_x0", "panels_x", "panels_x0", "panels_area", "panels_has_children",
           "panels_vertices", "panels_nest", "panels_children")


def _product_grid(level):
    parts, pans = grid.new_icos_grid(level)
    return dict(particles_x=parts.x, particles_x0=parts.x0, panels_x=pans.x, panels_x0=pans.x0,
                panels_area=pans.area, panels_has_children=pans.hasChildren.astype(np.int32),
                panels_vertices=pans.vertices, panels_nest=pans.nest, panels_children=pans.children)


@pytest.mark.parametrize("level", [0, 1, 2, 3, 4, 5, 6, 7])
def test_library_grid_equals_oracle_grid_bit_for_bit(level):
    """tc_icos_grid against the oracle's statement-for-statement restatement of InitIcosTriGrid /
    DivideTriPanel / TriPanelArea (oracle/icos_oracle.c): every position, Lagrangian coordinate,
    centre, area and index table identical, bit for bit."""
    from oracle import oracle as O

    ref = O.icos_grid(level)
    got = _product_grid(level)
    for k in _FIELDS:
        assert got[k].shape == ref[k].shape, k
        assert np.array_equal(got[k], ref[k]), k
    am, pm = O.gather_maps(ref["panels_has_children"])
    maps = grid.gather_maps(grid.new_icos_grid(level)[1])
    assert np.array_equal(maps.active, am) and np.array_equal(maps.passive, pm)


def test_oracle_grid_known_answers():
    """The oracle's grid on its own: PanelMax/ParticleMax counts, total area 4 pi, unit vectors."""
    from oracle import oracle as O

    for level in (0, 3, 6):
        g = O.icos_grid(level)
        npart, nedge, npan, nact = O.icos_sizes(level)
        assert (npart, npan, nact) == (2 + 10 * 4 ** level, sum(20 * 4 ** j for j in range(level + 1)),
                                        20 * 4 ** level)
        assert nedge == sum(30 * 4 ** j for j in range(level + 1))
        leaves = g["panels_has_children"] == 0
        assert np.count_nonzero(leaves) == nact
        assert abs(g["panels_area"][leaves].sum() - 4 * np.pi) < 1e-12
        np.testing.assert_allclose(np.linalg.norm(g["particles_x"], axis=1), 1.0, atol=1e-15)
    with pytest.raises(ValueError):
        O.icos_sizes(12)
