"""Seeded random problem shapes through the one-sum entry point against the oracle, every row:
source counts that are not multiples of the 256-source tile (from 1 up), target counts that are
not multiples of a CTA's targets, target ranges starting and ending inside tiles, all three target
classes, random subsets of a level-5 grid (sources from the panel centres, vertex and passive
targets from the vertices, so no target sits on a source) with random vorticity. FP64 within
1e-12, which checks the index logic exactly. FP32C within 1e-5: its error floor is eps * rho / h
(rho the radius of a CTA's patch of targets, h the distance to the nearest source); scattered
random points make rho large (a few hundred targets span much of the sphere) and h small (random
sets have close pairs), measured 1.9e-6 for 346 scattered targets among 257 scattered sources. The
FP32C bounds for grids are tested on full grids elsewhere, and an index error would show as an
O(1) error. Rows outside the range must be exactly zero."""
import numpy as np
import pytest

from oracle import oracle as O
from thesiscode_b200 import _native as N
from thesiscode_b200 import configs
from thesiscode_b200.panel_velocity import Context

pytestmark = pytest.mark.gpu
TOL = {"fp64": 1e-12, "fp32c": 1e-5}


def cases(seed=2024, count=16):
    g = configs.gaussian(level=5, delta=0.0)
    rng = np.random.default_rng(seed)
    for _ in range(count):
        n = int(rng.choice([1, 2, 255, 256, 257, int(rng.integers(3, 6000))]))
        cls = int(rng.integers(0, 3))
        x = np.ascontiguousarray(g.xA[rng.choice(g.nA, n, replace=False)])
        z = rng.standard_normal(n)
        a = rng.uniform(0.5, 1.5, n) * (4 * np.pi / max(n, 1))
        if cls == N.TC_ACTIVE:
            X, m = None, n
        else:
            m = int(rng.integers(1, 3000))
            X = np.ascontiguousarray(g.xV[rng.choice(g.nV, m, replace=False)])
        i0 = int(rng.integers(0, m))
        i1 = int(rng.integers(i0, m + 1))
        delta = float(rng.choice([0.0, 0.01, 0.05]))
        yield cls, X, x, z, a, m, i0, i1, delta


@pytest.mark.parametrize("prec", ["fp64", "fp32c"])
def test_random_shapes_against_oracle(gpu, prec):
    ctx = Context(0, prec)
    ctx.set_omega(2 * np.pi)
    worst = 0.0
    for cls, X, x, z, a, m, i0, i1, delta in cases():
        ctx.set_deltas(delta, delta, delta)
        dX, _ = ctx.velocity(cls, X, x, z, a, i0, i1)
        rows = np.arange(i0, i1, dtype=np.int32)
        assert np.all(dX[:i0] == 0) and np.all(dX[i1:] == 0), (cls, m, i0, i1)
        if rows.size == 0:
            continue
        ref = O.rows(cls, rows, X, x, z, a, delta=delta, nthreads=8)
        scale = max(np.abs(ref).max(), 1e-300)
        err = np.abs(dX[i0:i1] - ref).max() / scale
        worst = max(worst, err)
        assert err <= TOL[prec], (cls, x.shape[0], m, i0, i1, delta, err)
    ctx.close()
    assert worst < TOL[prec]
