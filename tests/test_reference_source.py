"""Parity against the reference's own code (no GPU).

The reference is Fortran and neither machine has a Fortran compiler, so its
hot path runs through oracle/f90, a translator of the Fortran 90 subset the
modules use, with strict IEEE double arithmetic. tests/golden/ref_*.npz hold
what the reference's statements computed (tests/golden/make_reference_fixtures.py):
its grid generator (NewGrid, ParticlesEdgesPanels2.f90:362-397), its initial
conditions, BVERK4 and StratosphereRK4 on 1-4 MPI ranks run as threads
(PanelVelocityParallel.f90:435-919), the three RHS sums (:1287-1412), the
Voronoi BVEVelocity and BVERK4 (VoronoiVelocityParallel.f90:300-515) and the
RH4 driver program's output; the serial twin (PanelVelocitySerial.f90) is run
live where the sources are.

Checked here, bit for bit: the C oracle (the checker of every GPU test) and
the library's host grid generator against those fixtures; the library's
initial-condition functions to rounding. Where the reference's sources are
present, the fixtures are regenerated from them and must be unchanged. The
translator's own semantics are tested on small Fortran programs written here.
"""
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from oracle.f90 import FortranSubsetError, Runner, rt
from oracle.f90 import reference as REF

GOLDEN = Path(__file__).resolve().parent / "golden"
DELTAS = (0.0, 0.0, 0.05)  # BVEActiveRHS, BVEPassiveRHS: none; BVESmoothVelocity: smooth = 0.05


@pytest.fixture(scope="module", autouse=True)
def _built(native_built):
    return native_built


def _load(name):
    return dict(np.load(GOLDEN / f"{name}.npz"))


def _state(f, prefix):
    n = len(prefix) + 1
    return {k[n:]: v for k, v in f.items() if k.startswith(prefix + "_")}


# ----------------------------------------------------------------------------- grid
def test_oracle_grid_equals_reference_grid():
    ref = _load("ref_grid_l3")
    g = O.icos_grid(3)
    for k, v in ref.items():
        assert np.array_equal(g[k], v), k


def test_library_host_grid_equals_reference_grid():
    from thesiscode_b200 import grid

    ref = _load("ref_grid_l3")
    parts, pans = grid.new_icos_grid(3)
    assert np.array_equal(parts.x, ref["particles_x"])
    assert np.array_equal(parts.x0, ref["particles_x0"])
    assert np.array_equal(pans.x, ref["panels_x"])
    assert np.array_equal(pans.x0, ref["panels_x0"])
    assert np.array_equal(pans.area, ref["panels_area"])
    assert np.array_equal(pans.hasChildren.astype(np.int32), ref["panels_has_children"])
    assert np.array_equal(pans.vertices, ref["panels_vertices"])
    assert np.array_equal(pans.nest, ref["panels_nest"])
    assert np.array_equal(pans.children, ref["panels_children"])


# ----------------------------------------------------------------------------- RK4 steps
@pytest.mark.parametrize("name", ["ref_bverk4_rh4_l2", "ref_bverk4_gauss_l2", "ref_bverk4_jet_l2",
                                  "ref_bverk4_rh4_l3"])
def test_oracle_bverk4_equals_reference(name):
    f = _load(name)
    s0, s1 = _state(f, "initial"), _state(f, "final")
    xV, xA, zA, xQ = s0["xV"], s0["xA"], s0["zetaA"], s0["xQ"]
    tke = []
    for _ in range(int(f["steps"])):
        xV, xA, zA, xQ, t, ke, relV = O.bve_rk4(xV, xA, zA, s0["areaA"], xQ, float(f["dt"]), 2 * np.pi,
                                                DELTAS, absVortV=s0["absVortV"])
        tke.append(t)
    assert np.array_equal(xV, s1["xV"])
    assert np.array_equal(xA, s1["xA"])
    assert np.array_equal(zA, s1["zetaA"])
    assert np.array_equal(xQ, s1["xQ"])
    assert np.array_equal(relV, s1["relVortV"])  # :651, relVort = absVort - 2 Omega z
    assert np.array_equal(np.array(tke), f["totalKE"])
    assert np.array_equal(ke, f["kineticEnergy"])


def test_oracle_stratosphere_step_equals_reference():
    f = _load("ref_strat_l2")
    s0, s1 = _state(f, "initial"), _state(f, "final")
    xV, xA, xQ = s0["xV"], s0["xA"], s0["xQ"]
    t = float(f["t0"])
    for _ in range(int(f["steps"])):
        xV, xA, relA, xQ, _, _, relV = O.strat_rk4(xV, xA, s0["absVortA"], s0["areaA"], xQ, t,
                                                   float(f["dt"]), absVortV=s0["absVortV"])
        t = t + float(f["dt"])
    assert np.array_equal(xV, s1["xV"])
    assert np.array_equal(xA, s1["xA"])
    assert np.array_equal(xQ, s1["xQ"])
    assert np.array_equal(relA, s1["zetaA"])
    assert np.array_equal(relV, s1["relVortV"])


def test_oracle_sums_equal_reference():
    f = _load("ref_rhs_l2")
    xA, zA, aA = f["xA"], f["zetaA"], f["areaA"]
    a0, a1 = f["active_range"]
    dx, dv = O.active_rhs(xA, zA, aA, int(a0), int(a1))
    assert np.array_equal(dx, f["active_dX"]) and np.array_equal(dv, f["active_dVort"])
    v0, v1 = f["vertex_range"]
    assert np.array_equal(O.passive_rhs(f["xV"], xA, zA, aA, int(v0), int(v1)), f["vertex_dX"])
    assert np.array_equal(O.smooth_velocity(f["xQ"], xA, zA, aA, 0.05, 0, len(f["xQ"])), f["passive_dX"])
    r0, r1 = f["voronoi_range"]
    out = O.voronoi_velocity(xA[:, 0], xA[:, 1], xA[:, 2], zA, aA, int(r0), int(r1),
                             dy=f["voronoi_dy0"], dz=f["voronoi_dz0"])
    for got, key in zip(out, ("voronoi_dx", "voronoi_dy", "voronoi_dz", "voronoi_dVort")):
        assert np.array_equal(got, f[key]), key


# ----------------------------------------------------------------------------- initial conditions
def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def test_library_initial_conditions_match_reference():
    """The library's restatements of the reference's vorticity functions (thesiscode_b200/ics.py)
    evaluate with numpy's transcendental functions, the reference with the C library's: equal to
    a few ulps of the largest value."""
    from thesiscode_b200 import ics

    s = _state(_load("ref_bverk4_rh4_l2"), "initial")
    assert _rel(ics.rh4_reference(s["xA"]), s["zetaA"]) < 1e-14
    assert _rel(ics.rh4_reference(s["xV"]), s["relVortV"]) < 1e-14
    s = _state(_load("ref_bverk4_gauss_l2"), "initial")
    zeta = ics.gaussian_reference(s["xA"])
    zeta = zeta - ics.remove_area_mean(zeta, s["areaA"])  # every leaf panel's area; divided ones are 0
    assert _rel(zeta, s["zetaA"]) < 1e-13
    s = _state(_load("ref_bverk4_jet_l2"), "initial")
    zeta = ics.jet_reference(s["xA"])
    zeta = zeta - ics.remove_area_mean(zeta, s["areaA"])
    assert _rel(zeta, s["zetaA"]) < 1e-13
    s = _state(_load("ref_strat_l2"), "initial")
    zeta = ics.stratosphere_rel_vort(s["xA"])
    zeta = zeta - ics.remove_area_mean(zeta, s["areaA"])
    assert _rel(zeta, s["zetaA"]) < 1e-13


# ----------------------------------------------------------------------------- fixtures vs source
needs_source = pytest.mark.skipif(not REF.available(), reason="the reference's sources are not on this machine")


@needs_source
def test_fixtures_regenerate_from_the_reference_source():
    g = REF.grid(3)
    for k, v in _load("ref_grid_l3").items():
        assert np.array_equal(g[k], v), k
    f = _load("ref_bverk4_rh4_l2")
    r = REF.bve_rk4(2, int(f["steps"]), float(f["dt"]), nprocs=int(f["nprocs"]), ic="rh4")
    for part in ("initial", "final"):
        for k, v in r[part].items():
            assert np.array_equal(v, f[f"{part}_{k}"]), (part, k)
    assert np.array_equal(r["totalKE"], f["totalKE"])


@needs_source
def test_reference_bverk4_is_independent_of_the_rank_count():
    """LoadBalance's row split (PanelVelocityParallel.f90:167-213) and the per-stage broadcasts
    leave every result bit for bit the same on 1, 2 and 5 ranks."""
    runs = [REF.bve_rk4(1, 1, 0.01, nprocs=p, ic="gauss") for p in (1, 2, 5)]
    for r in runs[1:]:
        for k, v in runs[0]["final"].items():
            assert np.array_equal(r["final"][k], v), k


# ----------------------------------------------------------------------------- translator semantics
_SEMANTICS = """
module KindsM
  implicit none
  integer, parameter :: KR = kind(0.d0)
end module KindsM

module SemM
  use KindsM
  implicit none
  private
  public Twice, run_ints, run_reals, run_arrays, run_calls, Counter
  real(KR), save :: hidden = 3.0_KR
  integer :: Counter = 0
  interface Twice
    module procedure TwiceInt
    module procedure TwiceReal
  end interface
contains
  function TwiceInt(i)
    integer, intent(in) :: i
    integer :: TwiceInt
    TwiceInt = 2*i
  end function
  function TwiceReal(x) result(y)
    real(KR), intent(in) :: x
    real(KR) :: y
    y = 2.0_KR*x
  end function
  subroutine Bump(k, by)
    integer, intent(inout) :: k
    integer, intent(in), optional :: by
    if (present(by)) then
      k = k + by
    else
      k = k + 1
    endif
    Counter = Counter + 1
  end subroutine
  subroutine run_ints(out)
    integer, intent(out) :: out(10)
    integer :: j, s
    out(1) = -7/2
    out(2) = mod(-7, 2)
    out(3) = modulo(-7, 2)
    out(4) = 2**10
    s = 0
    do j = 1, 10, 3
      s = s + j
    enddo
    out(5) = s
    out(6) = j
    do j = 10, 1, -4
      if (j == 6) cycle
      s = s - j
    enddo
    out(7) = s
    select case (s)
      case (:0)
        out(8) = -1
      case (1:20)
        out(8) = 1
      case default
        out(8) = 2
    end select
    out(9) = Twice(21)
    out(10) = int(-2.7_KR) + nint(2.5_KR) + nint(-2.5_KR)
  end subroutine
  subroutine run_reals(out)
    real(KR), intent(out) :: out(6)
    real(KR) :: v(3)
    v = [0.1_KR, 0.2_KR, 0.3_KR]
    out(1) = sum(v)
    out(2) = 0.1
    out(3) = (1.5_KR)**3
    out(4) = -2.0_KR**2
    out(5) = Twice(hidden)
    out(6) = dot_product(v, v)
  end subroutine
  subroutine run_arrays(a, b)
    integer, intent(inout) :: a(:,:)
    integer, allocatable, intent(out) :: b(:)
    integer :: j
    a(2, :) = a(1, :) * 10
    a(:, 1:3:2) = -a(:, 1:3:2)
    allocate(b(0:4))
    do j = lbound(b, 1), ubound(b, 1)
      b(j) = j*j
    enddo
    b(4:0:-2) = b(0:4:2) + 100
  end subroutine
  subroutine run_calls(k, arr)
    integer, intent(inout) :: k
    integer, intent(inout) :: arr(:)
    call Bump(k)
    call Bump(k, by=5)
    call Bump(arr(2), 7)
  end subroutine
end module SemM
"""


@pytest.fixture(scope="module")
def semantics(tmp_path_factory):
    src = tmp_path_factory.mktemp("f90") / "sem.f90"
    src.write_text(_SEMANTICS)
    r = Runner([src], [("semm", "run_ints"), ("semm", "run_reals"), ("semm", "run_arrays"),
                       ("semm", "run_calls")])
    return r.instance()


def test_translator_integer_semantics(semantics):
    out = rt.FArr(np.zeros(10, dtype=np.int64))
    semantics.proc("semm", "run_ints")(out)
    # -7/2 truncates; mod takes the dividend's sign, modulo the divisor's; the DO variable ends
    # one step past the last value; CYCLE skips; CASE ranges; generic resolved by type
    s = 1 + 4 + 7 + 10
    s2 = s - 10 - 2
    assert out.a.tolist() == [-3, -1, 1, 1024, s, 13, s2, 1, 42, -2 + 3 - 3]


def test_translator_real_semantics(semantics):
    out = rt.FArr(np.zeros(6))
    semantics.proc("semm", "run_reals")(out)
    assert out.a[0] == (0.0 + 0.1) + 0.2 + 0.3          # SUM left to right from 0
    assert out.a[1] == float(np.float32(0.1))             # default-kind literal
    assert out.a[2] == (1.5 * 1.5) * 1.5                  # integer power by multiplication
    assert out.a[3] == -4.0                               # -a**b is -(a**b)
    assert out.a[4] == 6.0                                # private module variable, generic
    assert out.a[5] == (0.0 + 0.1 * 0.1) + 0.2 * 0.2 + 0.3 * 0.3


def test_translator_arrays_and_bounds(semantics):
    a = rt.FArr(np.asfortranarray(np.arange(1, 7, dtype=np.int64).reshape(2, 3, order="F")))
    r = semantics.proc("semm", "run_arrays")(a, None)
    assert a.a.tolist() == [[-1, 3, -5], [-10, 30, -50]]
    b = r[1]
    assert b.lb == (0,)
    assert b.a.tolist() == [16 + 100, 1, 4 + 100, 9, 0 + 100]


def test_translator_arguments_by_reference(semantics):
    arr = rt.FArr(np.array([1, 2, 3], dtype=np.int64))
    r = semantics.proc("semm", "run_calls")(5, arr)
    assert r[0] == 5 + 1 + 5                      # scalar dummy written back
    assert arr.a.tolist() == [1, 9, 3]            # array element actual written back
    assert semantics.mod("semm").counter == 3     # module variable shared by the calls


def test_translator_refuses_constructs_outside_the_subset(tmp_path):
    src = tmp_path / "bad.f90"
    src.write_text("module BadM\ncontains\nsubroutine s(x)\n  real(8) :: x\n  go to 10\n"
                   "10 x = 1\nend subroutine\nend module BadM\n")
    with pytest.raises(FortranSubsetError):
        Runner([src], [("badm", "s")])


@needs_source
@pytest.mark.parametrize("ic", ["rh4", "jet"])
def test_oracle_equals_the_reference_serial_module(ic):
    """The serial twin PanelVelocitySerial.f90:272-557 (its own copies of the three sums): the same
    step as the parallel module, bit for bit, except that it leaves the particles' relVort as it
    was (the parallel module's :651 update is missing from it)."""
    r = REF.serial_bve_rk4(1, 2, 0.01, ic=ic)
    s0, s1 = r["initial"], r["final"]
    xV, xA, zA, xQ = s0["xV"], s0["xA"], s0["zetaA"], s0["xQ"]
    tke = []
    for _ in range(2):
        xV, xA, zA, xQ, t, ke, _ = O.bve_rk4(xV, xA, zA, s0["areaA"], xQ, 0.01, 2 * np.pi, DELTAS)
        tke.append(t)
    for got, key in ((xV, "xV"), (xA, "xA"), (zA, "zetaA"), (xQ, "xQ")):
        assert np.array_equal(got, s1[key]), key
    assert np.array_equal(np.array(tke), r["totalKE"])
    assert np.array_equal(ke, r["kineticEnergy"])
    assert np.array_equal(s1["relVortV"], s0["relVortV"])


@needs_source
def test_vtk_fixture_regenerates_from_the_reference_source():
    f = _load("ref_vtk_l1")
    v = REF.vtk_output(1)
    assert v["text"] == str(f["text"])
    for k, val in v.items():
        if k != "text":
            assert np.array_equal(val, f[k]), k


def test_translator_formatted_output():
    """The formatter behind WRITE: edit descriptors, groups, format reversion, the optional
    leading zero of F, overflow asterisks and gfortran's list-directed layout."""
    assert rt.fformat("(A,I0.2,A)", ["K", 7, ":"]) == ["K07:"]
    assert rt.fformat("(2(I3,1X),A4)", [1, -2, "abcdef"]) == ["  1  -2 abcd"]
    assert rt.fformat("(F5.3)", [0.5]) == ["0.500"]
    assert rt.fformat("(F4.3)", [0.5]) == [".500"]
    assert rt.fformat("(F4.1)", [-123.0]) == ["****"]
    assert rt.fformat("(I2)", [123]) == ["**"]
    assert rt.fformat("(F6.2)", [1.0, 2.0]) == ["  1.00", "  2.00"]  # reversion: one record each
    assert rt.fformat("('x=',F4.1,/,'y')", [1.0]) == ["x= 1.0", "y"]
    assert rt.fformat(None, ["a", "b", 5]) == [" ab           5"]
    with pytest.raises(NotImplementedError):
        rt.fformat("(E12.4)", [1.0])
