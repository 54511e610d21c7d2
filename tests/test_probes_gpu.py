"""The throughput probes behind the roofline figures (tc_probe_peak).

The pair-loop probe runs the FP32C kernel's own far-form step
(sp_far_run: per source pair and target one FADD2, six FFMA2 and two MUFU
reciprocals) over a resident shared-memory tile. Each pair needs one MUFU
reciprocal, so its rate cannot exceed the MUFU probe's. The kernel, which also
stages tiles, tests far/near and flushes, cannot exceed the probe's rate
either (up to timing noise). Bad arguments are refused."""
import ctypes

import numpy as np
import pytest

from thesiscode_b200 import _native as N
from thesiscode_b200 import configs
from thesiscode_b200.panel_velocity import Context

pytestmark = pytest.mark.gpu


def probe(kind, iters):
    v = ctypes.c_double()
    N.call("tc_probe_peak", 0, kind, iters, ctypes.byref(v))
    return v.value


def test_pair_loop_probe_is_bounded_by_the_mufu_pipe_and_bounds_the_kernel(gpu):
    far = max(probe(N.TC_PROBE_FAR_PAIRS, 512) for _ in range(3))
    rcp = max(probe(N.TC_PROBE_RCP32, 4096) for _ in range(3))
    assert 0.0 < far <= rcp * 1.01, (far, rcp)
    # the level-7 Gaussian active sum through the FP32C kernel, timed on the device
    w = configs.gaussian(level=7, delta=0.01)
    ctx = Context(0, "fp32c")
    ctx.set_deltas(*w.deltas)
    N.call("tc_stats_enable_timing", ctx.handle, 1)
    ctx.velocity(N.TC_ACTIVE, None, w.xA, w.zetaA, w.areaA)  # warm-up
    L, PL, PI, ms = (ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong(),
                     ctypes.c_double())
    N.call("tc_stats", ctx.handle, 1, ctypes.byref(L), ctypes.byref(PL), ctypes.byref(PI),
           ctypes.byref(ms))
    ctx.velocity(N.TC_ACTIVE, None, w.xA, w.zetaA, w.areaA)
    N.call("tc_stats", ctx.handle, 0, ctypes.byref(L), ctypes.byref(PL), ctypes.byref(PI),
           ctypes.byref(ms))
    ctx.close()
    rate = PI.value / (ms.value * 1e-3)
    assert PI.value == w.nA * (w.nA - 1)
    assert 0.5 * far < rate <= far * 1.02, (rate, far)


@pytest.mark.parametrize("kind,iters", [(-1, 16), (N.TC_PROBE_FAR_PAIRS + 1, 16),
                                        (N.TC_PROBE_FAR_PAIRS, 0), (N.TC_PROBE_FAR_PAIRS, 1 << 23)])
def test_probe_refuses_bad_arguments(gpu, kind, iters):
    v = ctypes.c_double()
    assert N.lib().tc_probe_peak(0, kind, iters, ctypes.byref(v)) == N.TC_ERR_ARG
