"""Batched ensembles (tc_batch_rk4): every instance of a batch evolves exactly as its own RK4 run
(checked against the oracle per instance), the CUDA-graph replay equals eager launches, and the
autotuner's choice is a valid variant."""
import numpy as np
import pytest

from oracle import oracle as O
from thesiscode_b200 import configs
from thesiscode_b200.batch import batch_info, batch_rk4
from thesiscode_b200.panel_velocity import Context

pytestmark = pytest.mark.gpu
TOL = {"fp64": 1e-12, "fp32c": 5e-7}  # levels 1-3: the coarse-grid FP32C bound


def small_batch(seed=4):
    ws = configs.batched_gaussians(count=6, seed=seed, levels=(1, 2, 3))
    ws[2].xV = np.zeros((0, 3))  # an instance without vertex targets
    return ws


@pytest.mark.parametrize("prec", ["fp64", "fp32c"])
def test_batch_instances_match_oracle(prec, gpu):
    ws = small_batch()
    ref = [w.copy() for w in ws]
    ctx = Context(0, prec)
    ctx.set_omega(ws[0].omega)
    ctx.set_deltas(*ws[0].deltas)
    nsteps, dt = 3, 0.01
    tke = batch_rk4(ctx, ws, dt, nsteps)
    for b, (w, r) in enumerate(zip(ws, ref)):
        xV, xA, zA = r.xV, r.xA, r.zetaA
        kes = []
        for _ in range(nsteps):
            xV, xA, zA, _, k, _, _ = O.bve_rk4(xV, xA, zA, r.areaA, np.zeros((0, 3)), dt, r.omega, r.deltas)
            kes.append(k)
        scale = np.abs(xA - r.xA).max()
        assert np.abs(w.xA - xA).max() <= TOL[prec] * scale, b
        assert np.abs(w.zetaA - zA).max() <= TOL[prec] * np.abs(zA - r.zetaA).max(), b
        if r.nV:
            assert np.abs(w.xV - xV).max() <= TOL[prec] * np.abs(xV - r.xV).max(), b
        np.testing.assert_allclose(tke[:, b], kes, rtol=2 * TOL[prec])
    info = batch_info(ctx)
    assert info["variant"] >= 0 and info["chunk_len"] in (1024, 2048, 4096, 8192) and info["work_items"] > 0
    ctx.close()


def test_graph_replay_equals_eager_launches(gpu):
    a, b = small_batch(seed=7), small_batch(seed=7)
    for graph, ws in ((True, a), (False, b)):
        ctx = Context(0, "fp32c")
        ctx.set_omega(ws[0].omega)
        ctx.set_deltas(*ws[0].deltas)
        batch_rk4(ctx, ws, 0.01, 2, graph=graph, autotune=False)
        batch_rk4(ctx, ws, 0.01, 2, graph=graph, autotune=False)  # second call replays the graph
        ctx.close()
    for wa, wb in zip(a, b):
        np.testing.assert_array_equal(wa.xA, wb.xA)
        np.testing.assert_array_equal(wa.zetaA, wb.zetaA)
        np.testing.assert_array_equal(wa.xV, wb.xV)


def test_batch_kernel_every_form_matches_oracle(gpu):
    """The persistent batch kernel with one variant of every FP32C form in the variant table
    (register or shared-memory accumulators, hi/lo near offsets, far-tile flush lengths),
    autotuning off: one RK4 step of each instance matches the oracle within the coarse-grid
    bound (5e-7)."""
    import ctypes

    from thesiscode_b200 import _native as N

    cnt = ctypes.c_int()
    N.call("tc_pair_variant_count", N.TC_FP32C, ctypes.byref(cnt))
    first_of_form = {}
    for v in range(cnt.value):
        info = (ctypes.c_int * 8)()
        N.call("tc_pair_variant_info", N.TC_FP32C, v, info)
        first_of_form.setdefault(info[7], v)
    assert len(first_of_form) >= 6
    ref0 = small_batch(seed=9)
    expect = []
    for r in ref0:
        xV, xA, zA, *_ = O.bve_rk4(r.xV, r.xA, r.zetaA, r.areaA, np.zeros((0, 3)), 0.01, r.omega, r.deltas)
        expect.append((xA, zA, xV))
    for form, v in sorted(first_of_form.items()):
        ws = [w.copy() for w in ref0]
        ctx = Context(0, "fp32c")
        ctx.set_omega(ws[0].omega)
        ctx.set_deltas(*ws[0].deltas)
        N.call("tc_set_pair_variant", ctx.handle, N.TC_FP32C, v)
        batch_rk4(ctx, ws, 0.01, 1, graph=False, autotune=False)
        assert batch_info(ctx)["variant"] == v
        ctx.close()
        assert form & 8, (form, v)
        tol = TOL["fp32c"]
        for b, (w, r, (xA, zA, xV)) in enumerate(zip(ws, ref0, expect)):
            scale = np.abs(xA - r.xA).max()
            assert np.abs(w.xA - xA).max() <= tol * scale, (form, v, b)
            assert np.abs(w.zetaA - zA).max() <= tol * np.abs(zA - r.zetaA).max(), (form, v, b)
