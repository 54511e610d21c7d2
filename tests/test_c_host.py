"""The C ABI from compiled C host programs: tests/c_host/bve_driver.c (one rank, the way a
Fortran BVE driver calls BVERK4) and tests/c_host/bve_sharded.c (ranks as threads, each computing
its LoadBalance rows of every RK4 stage and exchanging the packed source rows through host memory,
the sequence an MPI host runs with MPI_Allgatherv). The first also round-trips a checkpoint
(tc_rk4_save / tc_rk4_restore). Both build with gcc against
include/thesiscode_b200.h and link libthesiscode_b200.so like a Fortran or C driver would; on a
machine without a GPU they fail cleanly with the library's CUDA status. On the GPU the sharded
run matches the serial oracle."""
import os
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "c_host" / "bve_driver.c"
SHARDED = ROOT / "tests" / "c_host" / "bve_sharded.c"


def build_driver(tmp_path, native_built, src=SRC):
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("gcc not available")
    lib_dir = ROOT / "thesiscode_b200" / "_lib"
    exe = tmp_path / src.stem
    subprocess.run([gcc, "-O2", "-std=c11", "-pthread", f"-I{ROOT / 'include'}", str(src), "-o", str(exe),
                    f"-L{lib_dir}", "-lthesiscode_b200", f"-Wl,-rpath,{lib_dir}", "-lm"], check=True)
    return exe


def run_sharded(exe, tmp_path, w, nsteps, precision, nranks):
    """Writes the workload, runs the sharded driver, returns (rc, stderr, outputs or None)."""
    inp, out = tmp_path / "in.bin", tmp_path / "out.bin"
    np.concatenate([w.xA.ravel(), w.zetaA, w.areaA, w.xV.ravel(), w.xQ.ravel()]).tofile(inp)
    args = [str(exe), str(inp), str(out), str(w.nA), str(w.nV), str(w.nQ), str(nsteps), str(precision),
            str(nranks), repr(w.dt), repr(w.omega), *(repr(d) for d in w.deltas)]
    r = subprocess.run(args, capture_output=True, text=True, timeout=600)
    if r.returncode != 0:
        return r.returncode, r.stderr, None
    v = np.fromfile(out)
    nA, nV, nQ = w.nA, w.nV, w.nQ
    cuts = np.cumsum([3 * nA, nA, 3 * nV, 3 * nQ])
    xA, zA, xV, xQ, tke = np.split(v, cuts)
    return 0, r.stderr, (xA.reshape(nA, 3), zA, xV.reshape(nV, 3), xQ.reshape(nQ, 3), tke)


def test_c_driver_builds_and_fails_cleanly_without_gpu(tmp_path, native_built):
    import torch

    exe = build_driver(tmp_path, native_built)
    if torch.cuda.is_available():
        pytest.skip("a GPU is present: the GPU test runs the driver")
    r = subprocess.run([str(exe), "2", "1", "0"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 3, (r.returncode, r.stdout, r.stderr)
    assert "tc_create" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_c_driver_runs_bve_steps(tmp_path, native_built, gpu, precision):
    exe = build_driver(tmp_path, native_built)
    r = subprocess.run([str(exe), "4", "5", str(precision), str(tmp_path / "run.tcb")],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    assert "5120 active panels" in r.stdout
    assert "checkpoint round trip after 2 of 5 steps: identical" in r.stdout


def test_sharded_c_driver_builds_and_fails_cleanly_without_gpu(tmp_path, native_built):
    import torch

    from thesiscode_b200 import configs

    exe = build_driver(tmp_path, native_built, SHARDED)
    if torch.cuda.is_available():
        pytest.skip("a GPU is present: the GPU test runs the sharded driver")
    w = configs.rh4(level=2, parity=True, dt=0.01)
    rc, err, _ = run_sharded(exe, tmp_path, w, 1, 0, 2)
    assert rc == 3, (rc, err)  # every rank stops at its first CUDA error, none waits forever


@pytest.mark.gpu
@pytest.mark.parametrize("precision,nranks", [(0, 2), (0, 3), (1, 2)])
def test_sharded_c_driver_matches_serial_oracle(tmp_path, native_built, gpu, precision, nranks):
    """Level 4, parity mode (active panels delta 0, vertices delta 0, divided panels delta 0.05),
    two RK4 steps on 2 or 3 ranks (3: ragged LoadBalance chunks) against two serial oracle BVERK4
    steps: FP64 within 1e-12, FP32C within its level-4 bound 3e-7."""
    from oracle import oracle as O
    from thesiscode_b200 import configs

    exe = build_driver(tmp_path, native_built, SHARDED)
    w = configs.rh4(level=4, parity=True, dt=0.01)
    nsteps = 2
    rc, err, got = run_sharded(exe, tmp_path, w, nsteps, precision, nranks)
    assert rc == 0, err
    xA, zA, xV, xQ, tke = got
    rV, rA, rz, rQ = w.xV, w.xA, w.zetaA, w.xQ
    kes = []
    for _ in range(nsteps):
        rV, rA, rz, rQ, k, _, _ = O.bve_rk4(rV, rA, rz, w.areaA, rQ, w.dt, w.omega, w.deltas,
                                            nthreads=os.cpu_count() or 1)
        kes.append(k)
    tol = 1e-12 if precision == 0 else 3e-7

    def rel(a, b, a0):
        return np.abs(a - b).max() / np.abs(b - a0).max()

    assert rel(xA, rA, w.xA) <= tol
    assert rel(zA, rz, w.zetaA) <= tol
    assert rel(xV, rV, w.xV) <= tol
    assert rel(xQ, rQ, w.xQ) <= tol
    np.testing.assert_allclose(tke, kes, rtol=2 * tol)
