"""The checkpoint file format, on the CPU: the library's reader (tc_rk4_checkpoint_info, no GPU
needed) accepts a file written here from the documented layout, with its own FNV-1a hash, and
refuses truncated, corrupted, foreign or later-version files; thesiscode_b200.checkpoint.read
gives back the arrays written. The GPU tests check that tc_rk4_save writes this layout."""
import struct

import numpy as np
import pytest

from thesiscode_b200 import _native as N
from thesiscode_b200 import checkpoint as C


def fnv1a(data: bytes) -> int:
    h = 1469598103934665603
    for b in data:
        h = ((h ^ b) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


def write(path, xA, zA, aA, xV, xQ, omega=6.25, deltas=(0.0, 0.0, 0.05), steps=7, forced=None):
    arrays = [np.ascontiguousarray(a, dtype="<f8").ravel() for a in (xA, zA, aA, xV, xQ)]
    t0, fstep, dt = 0.0, 0, 0.0
    if forced is not None:
        absA, absV, t0, fstep, dt = forced
        arrays += [np.asarray(absA, "<f8"), np.asarray(absV, "<f8")]
    head = struct.pack("<8sIIiiiiqq6d", b"TCB2RK4\0", 1, int(forced is not None), len(zA), len(xV),
                       len(xQ), 1, steps, fstep, omega, *deltas, t0, dt)
    body = head + b"".join(a.tobytes() for a in arrays)
    path.write_bytes(body + struct.pack("<Q", fnv1a(body)))
    return body


@pytest.fixture
def state():
    rng = np.random.default_rng(5)
    return (rng.standard_normal((40, 3)), rng.standard_normal(40), rng.random(40),
            rng.standard_normal((22, 3)), rng.standard_normal((10, 3)))


def test_library_reads_a_file_written_from_the_layout(tmp_path, native_built, state):
    p = tmp_path / "a.tcb"
    write(p, *state)
    assert C.info(p) == {"nA": 40, "nV": 22, "nQ": 10, "forced": False, "steps": 7}
    r = C.read(p)
    for k, a in zip(("xA", "zetaA", "areaA", "xV", "xQ"), state):
        np.testing.assert_array_equal(r[k], a)
    assert r["omega"] == 6.25 and r["deltas"] == (0.0, 0.0, 0.05) and r["precision"] == 1
    q = tmp_path / "f.tcb"
    write(q, *state, forced=(np.arange(40.0), np.arange(22.0), 3.9, 2, 0.03))
    r = C.read(q)
    assert r["forced"] and r["t0"] == 3.9 and r["forced_step"] == 2 and r["dt"] == 0.03
    np.testing.assert_array_equal(r["absVortV"], np.arange(22.0))


def test_library_refuses_bad_files(tmp_path, native_built, state):
    good = tmp_path / "good.tcb"
    body = write(good, *state)
    raw = good.read_bytes()
    bad = {
        "truncated": raw[:-9],
        "short": raw[:50],
        "flipped": raw[:300] + bytes([raw[300] ^ 4]) + raw[301:],
        "magic": b"TCB2RK5\0" + raw[8:],
        "version": raw[:8] + (2).to_bytes(4, "little") + raw[12:],
        "flags": raw[:12] + (2).to_bytes(4, "little") + raw[16:],
        "sizes": raw[:16] + (41).to_bytes(4, "little") + raw[20:],
        "checksum": body + struct.pack("<Q", fnv1a(body) ^ 1),
    }
    for name, content in bad.items():
        p = tmp_path / f"{name}.tcb"
        p.write_bytes(content)
        with pytest.raises(N.TcError) as e:
            C.info(p)
        assert e.value.status == N.TC_ERR_ARG, name
    with pytest.raises(N.TcError):
        C.info(tmp_path / "missing.tcb")
