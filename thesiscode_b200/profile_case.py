"""One launch of the pair kernels on a workload of a chosen size, for profilers.

    python -m thesiscode_b200.profile_case --precision fp32c --level 6 [--what velocity|rk4]

`velocity` runs one TC_ACTIVE and one TC_VERTEX sum (two pair-kernel launches);
`rk4` runs one fused RK4 step (four pair-kernel launches). The Gaussian-vortex
workload with delta 0.01 is used at every level.
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
    ap.add_argument("--what", default="velocity", choices=["velocity", "rk4"])
    a = ap.parse_args()
    w = configs.gaussian(level=a.level, delta=0.01)
    ctx = Context(0, a.precision)
    ctx.set_omega(w.omega)
    ctx.set_deltas(*w.deltas)
    if a.what == "velocity":
        ctx.velocity(N.TC_ACTIVE, None, w.xA, w.zetaA, w.areaA)
        ctx.velocity(N.TC_VERTEX, w.xV, w.xA, w.zetaA, w.areaA)
    else:
        ctx.rk4_step(w.xA.copy(), w.zetaA.copy(), w.areaA, w.xV.copy(), w.xQ.copy(), w.dt, 1)
    ctx.synchronize()
    ctx.close()
    print(f"profile_case {a.precision} level {a.level} {a.what}: ok")


if __name__ == "__main__":
    main()
