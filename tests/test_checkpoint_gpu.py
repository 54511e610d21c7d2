"""Checkpoint and restart of the device-resident RK4 state (tc_rk4_save / tc_rk4_restore).

A run that stops after some steps, writes a checkpoint and continues in a fresh
context from that file must end bit for bit where the uninterrupted run ends.
Checked for the BVE step with all three target classes, in FP64 and FP32C
(the FP32C visiting order is rebuilt from the restored positions), and for the
forced model, whose clock (t0, step count, step length) travels in the file. A
missing, truncated or corrupted file is refused with TC_ERR_ARG and the
context keeps its state.
"""
import numpy as np
import pytest

from thesiscode_b200 import _native as N
from thesiscode_b200 import checkpoint, configs
from thesiscode_b200.panel_velocity import Context

pytestmark = pytest.mark.gpu


def _ctx(prec, w):
    ctx = Context(0, prec)
    ctx.set_omega(w.omega)
    ctx.set_deltas(*w.deltas)
    return ctx


@pytest.mark.parametrize("prec", ["fp64", "fp32c"])
def test_restart_from_checkpoint_continues_bit_for_bit(prec, gpu, tmp_path):
    w = configs.rh4(level=4, parity=True)  # active panels, vertices and divided panels
    dt, total, first = 0.01, 5, 2
    ctx = _ctx(prec, w)
    ctx.rk4_load(w.xA, w.zetaA, w.areaA, w.xV, w.xQ)
    tke_all = ctx.rk4_advance(dt, total)
    straight = ctx.rk4_store(w.nA, w.nV, w.nQ)
    ctx.close()

    ctx = _ctx(prec, w)
    ctx.rk4_load(w.xA, w.zetaA, w.areaA, w.xV, w.xQ)
    tke_a = ctx.rk4_advance(dt, first)
    path = tmp_path / "state.tcb"
    ctx.save_state(path)
    saved = ctx.rk4_store(w.nA, w.nV, w.nQ)
    ctx.close()
    # the file holds the documented layout (read back here, validated by the library's reader)
    r = checkpoint.read(path)
    assert r["steps"] == first and r["omega"] == w.omega and r["deltas"] == tuple(w.deltas)
    for k, a in zip(("xA", "zetaA", "xV", "xQ"), saved):
        np.testing.assert_array_equal(r[k], a)
    np.testing.assert_array_equal(r["areaA"], w.areaA)

    ctx = Context(0, prec)  # default Omega and deltas: the checkpoint sets them
    ctx.restore_state(path)
    assert ctx.get_omega() == w.omega and ctx.get_deltas() == tuple(w.deltas)
    assert ctx.steps_done() == first
    tke_b = ctx.rk4_advance(dt, total - first)
    resumed = ctx.rk4_store(w.nA, w.nV, w.nQ)
    assert ctx.steps_done() == total
    ctx.close()
    for a, b in zip(straight, resumed):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(np.concatenate([tke_a, tke_b]), tke_all)


def test_forced_run_restart_keeps_its_clock(gpu, tmp_path):
    w = configs.stratosphere(level=3, t0=3.9)  # across the forcing's ramp at t = 4
    dt, total, first = 0.03, 4, 2
    absA = w.meta["absVortA"]

    ctx = _ctx("fp64", w)
    s = w.copy()
    relA, _, tke_all, _ = ctx.strat_rk4_step(s.xA, absA, s.areaA, s.xV, s.xQ, 3.9, dt, total)
    ctx.close()

    ctx = _ctx("fp64", w)
    p = w.copy()
    ctx.strat_rk4_step(p.xA, absA, p.areaA, p.xV, p.xQ, 3.9, dt, first)
    path = tmp_path / "forced.tcb"
    ctx.save_state(path)
    ctx.close()

    ctx = Context(0, "fp64")
    ctx.restore_state(path)
    tke_b = ctx.rk4_advance(dt, total - first)
    xA, zA, xV, xQ = ctx.rk4_store(w.nA, w.nV, w.nQ)
    ctx.close()
    np.testing.assert_array_equal(xA, s.xA)
    np.testing.assert_array_equal(zA, relA)
    np.testing.assert_array_equal(xV, s.xV)
    np.testing.assert_array_equal(xQ, s.xQ)
    np.testing.assert_array_equal(tke_b, tke_all[first:])


def test_bad_checkpoints_are_refused_and_the_state_is_kept(gpu, tmp_path):
    w = configs.rh4(level=2, parity=True)
    ctx = _ctx("fp64", w)
    with pytest.raises(N.TcError) as e:
        ctx.save_state(tmp_path / "none.tcb")  # nothing loaded yet
    assert e.value.status == N.TC_ERR_STATE
    ctx.rk4_load(w.xA, w.zetaA, w.areaA, w.xV, w.xQ)
    ctx.rk4_advance(0.01, 1)
    good = tmp_path / "good.tcb"
    ctx.save_state(good)
    before = ctx.rk4_store(w.nA, w.nV, w.nQ)
    raw = good.read_bytes()
    bad = {
        "missing": None,
        "truncated": raw[:-9],
        "flipped": raw[:200] + bytes([raw[200] ^ 1]) + raw[201:],
        "magic": b"XXXXXXXX" + raw[8:],
        "version": raw[:8] + (2).to_bytes(4, "little") + raw[12:],
    }
    for name, content in bad.items():
        path = tmp_path / f"{name}.tcb"
        if content is not None:
            path.write_bytes(content)
        with pytest.raises(N.TcError) as e:
            ctx.restore_state(path)
        assert e.value.status == N.TC_ERR_ARG, name
        after = ctx.rk4_store(w.nA, w.nV, w.nQ)
        for a, b in zip(before, after):
            np.testing.assert_array_equal(a, b, err_msg=name)
    assert not (tmp_path / "good.tcb.tmp").exists()
    ctx.restore_state(good)
    for a, b in zip(before, ctx.rk4_store(w.nA, w.nV, w.nQ)):
        np.testing.assert_array_equal(a, b)
    ctx.close()
