"""The index-checked build (libthesiscode_b200_checked.so, TC_LIBRARY=checked).

compute-sanitizer cannot be run on these machines. Its stand-in is a build of
the same sources in which the hot-path kernels check every global-memory index
against its array's extent. Those kernels are the pair kernels (single and
batched), packing, the velocity and stage epilogues, and the adjoint's row
pass. An out-of-range
access is skipped and recorded, never performed. This file checks four things:

* The checks change no arithmetic. A fixed set of calls gives bit for bit the
  release build's results: velocity of every target class, RK4 steps with
  graph replay, the forced model, the allocation-free entry point, a
  batched ensemble and the adjoint, in both precisions. The record stays
  empty.
* The checks fire. For each site, the declared extent is capped below what
  the call touches, while the real arrays keep their size. The device's record
  then names that site, with an index at or past the cap. Once the cap is
  removed, the same context gives the uncapped result again and the record
  stays empty.
* The GPU parity suite runs clean under the checked build. The hot-path test
  files run in a child process with TC_LIBRARY=checked. After every test,
  conftest reads the record and fails the test if anything was recorded.
* The release build reports no checks (CPU).

The children run tests/bounds_cases.py and pytest, so each process loads
exactly one build of the library.
"""
import json
import os
import re
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from thesiscode_b200 import build as B

ROOT = Path(__file__).resolve().parents[1]
CASES = Path(__file__).resolve().parent / "bounds_cases.py"
# hot-path test files run again under the checked build
SUITE = ["test_parity_gpu.py", "test_random_sizes_gpu.py", "test_graph_gpu.py", "test_batch_gpu.py",
         "test_strat_gpu.py", "test_voronoi_gpu.py", "test_dist_gpu.py", "test_finite_checks_gpu.py",
         "test_reference_gpu.py", "test_fortran_shim_gpu.py", "test_configs_gpu.py",
         "test_adjoint_gpu.py", "test_zz_no_alloc.py"]


def _child(args, checked, timeout):
    env = dict(os.environ)
    env.pop("TC_LIBRARY", None)
    if checked:
        env["TC_LIBRARY"] = "checked"
    return subprocess.run([sys.executable, *args], cwd=ROOT, env=env, capture_output=True,
                          text=True, timeout=timeout)


@pytest.fixture(scope="module")
def both_built(native_built):
    B.build()
    B.build(checked=True)
    return True


def test_release_library_reports_no_checks(native_built):
    import ctypes

    from thesiscode_b200 import _native as N

    if N.CHECKED:
        pytest.skip("this process loaded the checked build")
    assert N.lib().tc_bounds_checked() == 0
    rec = (ctypes.c_longlong * 4)()
    assert N.lib().tc_bounds_status(0, rec, 0) == 0 and list(rec) == [0, 0, 0, 0]


def test_checked_library_exports_the_header(both_built):
    import ctypes

    from thesiscode_b200 import _native as N

    lib = ctypes.CDLL(str(B.lib_path(checked=True)))
    for name in N.SIGNATURES:
        assert hasattr(lib, name), name
    lib.tc_bounds_checked.restype = ctypes.c_int
    assert lib.tc_bounds_checked() == 1


@pytest.mark.gpu
def test_checked_build_gives_the_release_results_bit_for_bit(both_built, gpu, tmp_path):
    out = {}
    for checked in (False, True):
        path = tmp_path / f"results_{int(checked)}.npz"
        r = _child([str(CASES), "results", str(path)], checked, 600)
        assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
        out[checked] = dict(np.load(path))
    rel, chk = out[False], out[True]
    assert int(rel["checked"]) == 0 and int(chk["checked"]) == 1
    assert chk["record"][0] == 0, f"index check fired: {chk['record']}"
    assert set(rel) == set(chk)
    for k in rel:
        if k not in ("checked", "record"):
            assert np.all(np.isfinite(rel[k])), k
            np.testing.assert_array_equal(chk[k], rel[k], err_msg=k)


@pytest.mark.gpu
def test_capped_extents_are_recorded_and_the_context_recovers(both_built, gpu, tmp_path):
    path = tmp_path / "caps.json"
    r = _child([str(CASES), "caps", str(path)], True, 600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    report = json.loads(path.read_text())
    assert len(report) >= 20
    for c in report:
        what = f"{c['site']} {c['precision']} {c['case']}: {c}"
        assert c["clean_before"] == 0, what
        rec = c["record"]
        assert rec["count"] >= 1 and rec["site"] == c["site_id"], what
        assert rec["extent"] == c["cap"] and rec["index"] >= c["cap"], what
        assert c["clean_after"] == 0 and c["same_after"], what


@pytest.mark.gpu
def test_gpu_suite_runs_clean_under_the_checked_build(both_built, gpu):
    files = [f"tests/{f}" for f in SUITE]
    r = _child(["-m", "pytest", "-q", "-m", "gpu", "-p", "no:cacheprovider", *files], True, 1500)
    tail = r.stdout[-4000:] + r.stderr[-2000:]
    assert r.returncode == 0, tail
    m = re.search(r"(\d+) passed", r.stdout)
    assert m and int(m.group(1)) >= 100 and " failed" not in r.stdout, tail
