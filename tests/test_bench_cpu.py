"""bench.py's reference arm runs on the host alone and prints one JSON line with the keys the
benchmark contract asks for (on the small level-4 RH4 workload, a few seconds of CPU), and maps
only the oracle's libraries, none of the product's."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_reference_arm_prints_one_contract_line(native_built):
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "2",
                          "--warmup", "3", "--config", "rh4_l4"], capture_output=True, text=True,
                         timeout=600, check=True).stdout.strip().splitlines()
    assert len(out) == 1
    line = json.loads(out[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["steps"] == 2 and line["warmup"] == 3
    assert line["value"] > 0 and line["higher_is_better"] is True
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["value"] == line["value"] and cb["cores"] >= 1
    assert "x86-64-" in cb["build"] and "ifort -O2" in cb["build"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["value"] == line["value"]
    # the arm builds its inputs on the oracle's grid: the product library is never mapped
    libs = line["libraries_loaded"]
    assert libs and all(lib.startswith("oracle/_build/") for lib in libs), libs
