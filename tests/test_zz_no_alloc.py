"""The allocation-free velocity entry point (tc_bs_velocity_device_noalloc).

It exists for callers that cannot let the library allocate device memory in
the middle of their work - a host application whose device memory is owned by
its own pool, or a stepping loop that must not take cudaMalloc's implicit
device-wide synchronisation - and keeps its scratch in a fixed 32 MiB array
inside the library. This file is collected last so that a failure here never
stops the other tests from running; it passes alone in a fresh process too.

Checked through the C ABI against the allocating entry point
(tc_bs_velocity_device) on the same device arrays, within the tolerances the
parity tests use, on two calls in a row with different inputs (the second call
must not see the first call's leftovers); against the FP64 oracle, including
targets handed over in a shuffled order (the FP32C path keeps the library's
visiting order, so its accuracy does not depend on the caller's order); for
all three target classes; at a size just under the scratch limit, where the
space left caps the number of source chunks; and the size limit itself.
"""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O
from thesiscode_b200 import _native as N
from thesiscode_b200 import configs
from thesiscode_b200.panel_velocity import Context

pytestmark = pytest.mark.gpu
TOL = {"fp64": 1e-12, "fp32c": 3e-7}
# against the oracle: FP64 1e-12; FP32C the parity tests' stated bound at level 6
ORACLE_TOL = {"fp64": 1e-12, "fp32c": 2e-7}
SCRATCH = 32 << 20


def _dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _call(name, ctx, cls, dX, dx, dz, da, m, n, i0, i1):
    import torch

    u = torch.full((m, 3), np.nan, dtype=torch.float64, device="cuda")
    v = torch.full((m,), np.nan, dtype=torch.float64, device="cuda")
    N.call(name, ctx.handle, cls, _ptr(dX), m, _ptr(dx), _ptr(dz), _ptr(da), n, i0, i1, _ptr(u), _ptr(v))
    torch.cuda.synchronize()
    return u.cpu().numpy(), v.cpu().numpy()


def _both(ctx, cls, X, x, z, a, i0, i1):
    """Run the allocating and the allocation-free entry points on the same device arrays."""
    n = x.shape[0]
    m = n if cls == N.TC_ACTIVE else X.shape[0]
    dx, dz, da = _dev(x), _dev(z), _dev(a)
    dX = None if cls == N.TC_ACTIVE else _dev(X)
    return [_call(name, ctx, cls, dX, dx, dz, da, m, n, i0, i1)
            for name in ("tc_bs_velocity_device", "tc_bs_velocity_device_noalloc")]


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("prec", ["fp64", "fp32c"])
def test_no_alloc_matches_allocating_entry_point_twice(prec, gpu):
    ctx = Context(0, prec)
    w1 = configs.gaussian(level=5, delta=0.01)
    ctx.set_omega(w1.omega)
    ctx.set_deltas(*w1.deltas)
    # call 1: active panels, a partial target range
    (u_ref, v_ref), (u, v) = _both(ctx, N.TC_ACTIVE, None, w1.xA, w1.zetaA, w1.areaA, 1000, 17000)
    assert np.all(np.isfinite(u)) and np.all(np.isfinite(v))
    assert _rel(u, u_ref) <= TOL[prec]
    assert _rel(v, v_ref) <= TOL[prec]
    assert np.all(u[:1000] == 0) and np.all(u[17000:] == 0)
    # call 2: different sizes and class; the scratch still holds call 1's data
    w2 = configs.rh4(level=4, parity=True)
    ctx.set_omega(w2.omega)
    ctx.set_deltas(*w2.deltas)
    (u_ref, _), (u, _) = _both(ctx, N.TC_PASSIVE, w2.xQ, w2.xA, w2.zetaA, w2.areaA, 0, w2.nQ)
    assert np.all(np.isfinite(u))
    assert _rel(u, u_ref) <= TOL[prec]
    ctx.close()


@pytest.mark.parametrize("prec", ["fp64", "fp32c"])
def test_no_alloc_against_oracle_shuffled_vertices(prec, gpu):
    """Level-6 Gaussian, delta 0.01: active panels and the vertices in a seeded random order
    (not spatially coherent), both against the strict oracle on 2,048 seeded rows each."""
    w = configs.gaussian(level=6, delta=0.01)
    ctx = Context(0, prec)
    ctx.set_omega(w.omega)
    ctx.set_deltas(*w.deltas)
    rng = np.random.default_rng(61)
    xV = w.xV[rng.permutation(w.nV)]
    dx, dz, da = _dev(w.xA), _dev(w.zetaA), _dev(w.areaA)
    uA, _ = _call("tc_bs_velocity_device_noalloc", ctx, N.TC_ACTIVE, None, dx, dz, da, w.nA, w.nA, 0, w.nA)
    uV, _ = _call("tc_bs_velocity_device_noalloc", ctx, N.TC_VERTEX, _dev(xV), dx, dz, da, w.nV, w.nA, 0,
                  w.nV)
    ctx.close()
    ra = np.sort(rng.choice(w.nA, 2048, replace=False)).astype(np.int32)
    rv = np.sort(rng.choice(w.nV, 2048, replace=False)).astype(np.int32)
    refA = O.rows(0, ra, None, w.xA, w.zetaA, w.areaA, delta=0.01, nthreads=8)
    refV = O.rows(1, rv, xV, w.xA, w.zetaA, w.areaA, delta=0.01, nthreads=8)
    assert _rel(uA[ra], refA) <= ORACLE_TOL[prec]
    assert _rel(uV[rv], refV) <= ORACLE_TOL[prec]


@pytest.mark.parametrize("prec", ["fp64", "fp32c"])
def test_no_alloc_vertex_class_and_repeat(prec, gpu):
    """TC_VERTEX against the allocating entry point; then a call on other inputs and the first
    call again: the repeat gives bit for bit the first result (nothing carries over)."""
    w = configs.rh4(level=5, delta=0.0)
    ctx = Context(0, prec)
    ctx.set_omega(w.omega)
    ctx.set_deltas(*w.deltas)
    (u_ref, _), (u1, _) = _both(ctx, N.TC_VERTEX, w.xV, w.xA, w.zetaA, w.areaA, 0, w.nV)
    assert _rel(u1, u_ref) <= TOL[prec]
    g = configs.gaussian(level=4, delta=0.02)
    _both(ctx, N.TC_ACTIVE, None, g.xA, g.zetaA, g.areaA, 0, g.nA)
    (_, _), (u2, _) = _both(ctx, N.TC_VERTEX, w.xV, w.xA, w.zetaA, w.areaA, 0, w.nV)
    assert np.array_equal(u1, u2)
    ctx.close()


@pytest.mark.parametrize("prec", ["fp64", "fp32c"])
def test_no_alloc_near_the_scratch_limit(prec, gpu):
    """A vertex sum sized so the space left caps the source chunks: n = 262,144 sources (8 MiB)
    and m = 400,000 targets (9.6 MB of partial sums per chunk): FP64 has room for two chunks,
    FP32C (whose visiting order takes about 10 MB more) for one, where the allocating entry point
    is free to take more."""
    rng = np.random.default_rng(5)
    n, m = 262_144, 400_000

    def sphere(k):
        v = rng.standard_normal((k, 3))
        return v / np.linalg.norm(v, axis=1, keepdims=True)

    x, X = sphere(n), sphere(m)
    z = rng.standard_normal(n)
    a = np.full(n, 4 * np.pi / n)
    assert 32 * n + 24 * m < SCRATCH < 32 * n + 3 * 24 * m
    ctx = Context(0, prec)
    ctx.set_deltas(0.01, 0.01, 0.01)
    (u_ref, _), (u, _) = _both(ctx, N.TC_VERTEX, X, x, z, a, 0, m)
    assert np.all(np.isfinite(u))
    assert _rel(u, u_ref) <= TOL[prec]
    ctx.close()


def test_no_alloc_rejects_sizes_beyond_its_scratch(gpu):
    import torch

    ctx = Context(0, "fp64")
    n = 700_000  # 32*n + 24*n > 32 MiB; real buffers of that size, so nothing can be read past
    x = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    z = torch.zeros(n, dtype=torch.float64, device="cuda")
    u = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    v = torch.zeros(n, dtype=torch.float64, device="cuda")
    rc = N.lib().tc_bs_velocity_device_noalloc(ctx.handle, N.TC_ACTIVE, None, n, _ptr(x), _ptr(z),
                                               _ptr(z), n, 0, n, _ptr(u), _ptr(v))
    assert rc == N.TC_ERR_ARG
    assert b"32 MiB" in N.lib().tc_last_error()
    ctx.close()
