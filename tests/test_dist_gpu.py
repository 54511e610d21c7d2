"""The target-sharded driver (dist.py) with the library backend on the GPU: two ranks emulated
by two host threads, each with its own library context on the same GPU, exchanging source rows
through an in-process collective. No kernel waits on another (every exchange is a host-side
copy between the contexts' buffers), so the ranks need not run concurrently on the device.
Checked against the FP64 oracle's serial BVERK4 (PanelVelocityParallel.f90:435-658)."""
import threading

import numpy as np
import pytest
import torch

from oracle import oracle as O
from thesiscode_b200 import configs
from thesiscode_b200.dist import DistributedPanelVelocity, LibBackend

pytestmark = pytest.mark.gpu


class ThreadComm:
    """In-process all_gather / all_reduce / barrier for `world` rank threads."""

    ReduceOp = torch.distributed.ReduceOp

    def __init__(self, world):
        self.world = world
        self.sync = threading.Barrier(world, timeout=60)
        self.slots = [None] * world
        self.local = threading.local()

    def view(self, rank):
        comm = self

        class View:
            ReduceOp = ThreadComm.ReduceOp

            def get_rank(self, group=None):
                return rank

            def get_world_size(self, group=None):
                return comm.world

            def barrier(self, group=None):
                comm.sync.wait()

            def all_gather(self, out, t, group=None):
                torch.cuda.synchronize()
                comm.slots[rank] = t
                comm.sync.wait()
                for r in range(comm.world):
                    out[r].copy_(comm.slots[r])
                torch.cuda.synchronize()
                comm.sync.wait()

            def all_reduce(self, t, op=ThreadComm.ReduceOp.SUM, group=None):
                torch.cuda.synchronize()
                comm.slots[rank] = t.clone()
                comm.sync.wait()
                vals = torch.stack([s.to(t.device) for s in comm.slots])
                t.copy_(vals.max(0).values if op == ThreadComm.ReduceOp.MAX else vals.sum(0))
                torch.cuda.synchronize()
                comm.sync.wait()

        return View()


def run_ranks(w, precision, world=2, steps=2):
    comm = ThreadComm(world)
    out, errs = [None] * world, []

    def rank_main(r):
        try:
            drv = DistributedPanelVelocity(0, precision, backend=LibBackend(0, precision), comm=comm.view(r))
            drv.load(w)
            drv.advance(w.dt, steps)
            st = drv.store()
            st["tke"] = np.array(drv.totalKE)
            out[r] = st
            drv.close()
        except Exception as e:  # surfaced by the test
            errs.append(e)
            comm.sync.abort()

    threads = [threading.Thread(target=rank_main, args=(r,)) for r in range(world)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=300)
    assert not any(t.is_alive() for t in threads), "a rank thread hung"
    if errs:
        raise errs[0]
    return out


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32c", 5e-7)])
def test_two_rank_driver_matches_serial_oracle(gpu, precision, tol):
    w = configs.rh4(level=3, parity=True, dt=0.01)
    xV, xA, zA, xQ = w.xV, w.xA, w.zetaA, w.xQ
    tkes = []
    for _ in range(2):
        xV, xA, zA, xQ, tke, _, _ = O.bve_rk4(xV, xA, zA, w.areaA, xQ, w.dt, w.omega, w.deltas, nthreads=8)
        tkes.append(tke)
    res = run_ranks(w, precision)
    for st in res:
        assert np.abs(st["xA"] - xA).max() <= tol * np.abs(xA - w.xA).max()
        assert np.abs(st["xV"] - xV).max() <= tol * np.abs(xV - w.xV).max()
        assert np.abs(st["xQ"] - xQ).max() <= tol * np.abs(xQ - w.xQ).max()
        assert np.abs(st["zetaA"] - zA).max() <= tol * np.abs(zA - w.zetaA).max()
        np.testing.assert_allclose(st["tke"], tkes, rtol=2 * tol)
    # both ranks end with the same full state
    for k in ("xA", "zetaA", "xV", "xQ"):
        assert np.array_equal(res[0][k], res[1][k])
