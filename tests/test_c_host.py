"""The C ABI from a compiled C host program (tests/c_host/bve_driver.c): it builds with gcc
against include/thesiscode_b200.h and links libthesiscode_b200.so like a Fortran or C driver
would; on a machine without a GPU it must fail cleanly with the library's CUDA status."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "c_host" / "bve_driver.c"


def build_driver(tmp_path, native_built):
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("gcc not available")
    lib_dir = ROOT / "thesiscode_b200" / "_lib"
    exe = tmp_path / "bve_driver"
    subprocess.run([gcc, "-O2", "-std=c11", f"-I{ROOT / 'include'}", str(SRC), "-o", str(exe),
                    f"-L{lib_dir}", "-lthesiscode_b200", f"-Wl,-rpath,{lib_dir}", "-lm"], check=True)
    return exe


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
    r = subprocess.run([str(exe), "4", "5", str(precision)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    assert "5120 active panels" in r.stdout
