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
must not see the first call's leftovers), and the size limit.
"""
import ctypes

import numpy as np
import pytest

from thesiscode_b200 import _native as N
from thesiscode_b200 import configs
from thesiscode_b200.panel_velocity import Context

pytestmark = pytest.mark.gpu
TOL = {"fp64": 1e-12, "fp32c": 3e-7}


def _dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _both(ctx, cls, X, x, z, a, i0, i1):
    """Run the allocating and the allocation-free entry points on the same device arrays."""
    import torch

    n = x.shape[0]
    m = n if cls == N.TC_ACTIVE else X.shape[0]
    dx, dz, da = _dev(x), _dev(z), _dev(a)
    dX = None if cls == N.TC_ACTIVE else _dev(X)
    outs = []
    for name in ("tc_bs_velocity_device", "tc_bs_velocity_device_noalloc"):
        u = torch.full((m, 3), np.nan, dtype=torch.float64, device="cuda")
        v = torch.full((m,), np.nan, dtype=torch.float64, device="cuda")
        N.call(name, ctx.handle, cls, _ptr(dX), m, _ptr(dx), _ptr(dz), _ptr(da), n, i0, i1, _ptr(u),
               _ptr(v))
        torch.cuda.synchronize()
        outs.append((u.cpu().numpy(), v.cpu().numpy()))
    return outs


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
    assert b"32 MiB" in N.lib().tc_last_error() or b"scratch" in N.lib().tc_last_error()
    ctx.close()
