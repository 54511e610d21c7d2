"""One launch of the pair kernels on a workload of a chosen size, for profilers.

    python -m thesiscode_b200.profile_case --precision fp32c --level 6 \
        [--what velocity|rk4|adjoint|batch|strat|grid] [--variant ID]

`velocity` runs one TC_ACTIVE and one TC_VERTEX sum (two pair-kernel launches);
`rk4` runs one fused RK4 step (four pair-kernel launches); `adjoint` runs the
FP64 adjoint of two RK4 steps (eight vector-Jacobian pair launches); `batch`
runs one RK4 step of the 64-instance Gaussian ensemble (levels 3 to `--level`)
without autotuning or graph (four persistent batch-kernel launches); `strat`
runs one forced stratosphere RK4 step (parity mode); `grid` generates the
icosahedral grid of `--level` on the GPU (tc_icos_grid_device). The Gaussian-vortex
workload with delta 0.01 is used at every level for the first three.
`--variant` selects a pair-kernel variant of the chosen precision (default:
the library's default) for `velocity` and `rk4`.
"""
from __future__ import annotations

import argparse

from . import _native as N
from . import configs
from .panel_velocity import Context


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--precision", default="fp32c", choices=["fp32c", "fp64"])
    ap.add_argument("--level", type=int, default=6)
    ap.add_argument("--what", default="velocity",
                    choices=["velocity", "rk4", "adjoint", "batch", "strat", "grid"])
    ap.add_argument("--variant", type=int, default=None)
    a = ap.parse_args()
    if a.what in ("batch", "strat", "grid"):
        ctx = Context(0, a.precision)
        if a.what == "grid":
            from .grid import new_icos_grid_device

            new_icos_grid_device(ctx, a.level)
        elif a.what == "batch":
            from .batch import batch_rk4

            ws = configs.batched_gaussians(count=64, seed=4, levels=tuple(range(3, a.level + 1)))
            ctx.set_omega(ws[0].omega)
            ctx.set_deltas(*ws[0].deltas)
            batch_rk4(ctx, ws, ws[0].dt, 1, graph=False, autotune=False)
        else:
            w = configs.stratosphere(level=a.level, dt=0.01)
            ctx.set_omega(w.omega)
            ctx.set_deltas(*w.deltas)
            ctx.strat_rk4_step(w.xA.copy(), w.meta["absVortA"], w.areaA, w.xV.copy(), w.xQ.copy(),
                               w.meta["t0"], w.dt, 1, absVortV=w.meta["absVortV"])
        ctx.synchronize()
        ctx.close()
        print(f"profile_case {a.precision} level {a.level} {a.what}: ok")
        return
    w = configs.gaussian(level=a.level, delta=0.01)
    ctx = Context(0, a.precision)
    ctx.set_omega(w.omega)
    ctx.set_deltas(*w.deltas)
    if a.variant is not None:
        N.call("tc_set_pair_variant", ctx.handle, N.TC_FP64 if a.precision == "fp64" else N.TC_FP32C, a.variant)
    if a.what == "velocity":
        ctx.velocity(N.TC_ACTIVE, None, w.xA, w.zetaA, w.areaA)
        ctx.velocity(N.TC_VERTEX, w.xV, w.xA, w.zetaA, w.areaA)
    elif a.what == "rk4":
        ctx.rk4_step(w.xA.copy(), w.zetaA.copy(), w.areaA, w.xV.copy(), w.xQ.copy(), w.dt, 1)
    else:
        import numpy as np

        J, gz, gx = np.zeros(1), np.zeros(w.nA), np.zeros((w.nA, 3))
        N.call("tc_rk4_adjoint", ctx.handle, N.dptr(w.xA), N.dptr(w.zetaA), N.dptr(w.areaA), w.nA, w.dt, 2, 2,
               N.TC_J_ENSTROPHY, 0, N.dptr(J), N.dptr(gz), N.dptr(gx))
    ctx.synchronize()
    ctx.close()
    print(f"profile_case {a.precision} level {a.level} {a.what}: ok")


if __name__ == "__main__":
    main()
