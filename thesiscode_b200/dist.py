"""Target-sharded multi-rank RK4 (the reference's MPI scheme, on NCCL over NVLink).

PanelVelocityParallel.f90 replicates all data on every rank, splits the
target rows of each class into contiguous LoadBalance chunks (:167-213),
and after each RHS evaluation broadcasts every rank's rows to all others
(the per-stage MPI_BCAST loops, :476-489, :530-543, :572-585, :614-627).

Here each rank (one process per GPU) holds the full state once, computes
its rows of each stage on its GPU, and the only per-stage exchange is the
all-gather of the next stage's packed source rows {x, y, z, zeta*A} of the
active panels (32 B per panel). Vertex and divided-panel targets never
leave their rank until `store()` gathers the final state. The collective
goes through torch.distributed (NCCL on GPUs, gloo in CPU tests); the
stage arithmetic runs in libthesiscode_b200 (`LibBackend`).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from .panel_velocity import load_balance

SOURCES, XA, ZETA, XV, XQ, KE = range(6)
WIDTH = {SOURCES: 4, XA: 3, ZETA: 1, XV: 3, XQ: 3, KE: 1}


@dataclass
class Ranges:
    a: tuple[np.ndarray, np.ndarray]
    v: tuple[np.ndarray, np.ndarray]
    q: tuple[np.ndarray, np.ndarray]

    def rank(self, r: int) -> tuple[int, int, int, int, int, int]:
        return (int(self.a[0][r]), int(self.a[1][r]), int(self.v[0][r]), int(self.v[1][r]),
                int(self.q[0][r]), int(self.q[1][r]))


class LibBackend:
    """Stage primitives of libthesiscode_b200 on one GPU (device tensors via torch)."""

    def __init__(self, device: int, precision):
        import torch

        from .panel_velocity import Context

        self.torch = torch
        self.device = torch.device(f"cuda:{device}")
        self.ctx = Context(device, precision)
        self.ke_dev = torch.zeros(1, dtype=torch.float64, device=self.device)

    def bind_stream(self, stream) -> None:
        self.ctx.set_stream(stream.cuda_stream)

    def load(self, w) -> None:
        from . import _native as N

        self.n = (w.nA, w.nV, w.nQ)
        self.ctx.set_omega(w.omega)
        self.ctx.set_deltas(*w.deltas)
        N.call("tc_rk4_load", self.ctx.handle, N.dptr(w.xA), N.dptr(w.zetaA), N.dptr(w.areaA), w.nA,
               N.dptr(w.xV), w.nV, N.dptr(w.xQ) if w.nQ else None, w.nQ, 0)

    def pack_sources(self) -> None:
        from . import _native as N

        N.call("tc_rk4_pack_sources", self.ctx.handle)

    def stage(self, s: int, dt: float, rng: tuple) -> None:
        from . import _native as N

        ke = ctypes.c_void_p(self.ke_dev.data_ptr()) if s == 0 else None
        N.call("tc_rk4_stage_range", self.ctx.handle, s, float(dt), *rng, ke)

    def stage_ke(self):
        return self.ke_dev

    def empty(self, rows: int, width: int):
        return self.torch.empty((rows, width), dtype=self.torch.float64, device=self.device)

    def export_rows(self, which: int, r0: int, n: int, out) -> None:
        from . import _native as N

        N.call("tc_rk4_copy_rows", self.ctx.handle, which, r0, n, ctypes.c_void_p(out.data_ptr()), 0)

    def import_rows(self, which: int, r0: int, n: int, src) -> None:
        from . import _native as N

        N.call("tc_rk4_copy_rows", self.ctx.handle, which, r0, n, ctypes.c_void_p(src.data_ptr()), 1)

    def state(self) -> dict:
        from . import _native as N

        nA, nV, nQ = self.n
        out = dict(xA=np.zeros((nA, 3)), zetaA=np.zeros(nA), xV=np.zeros((nV, 3)), xQ=np.zeros((nQ, 3)),
                   ke=np.zeros(nA))
        N.call("tc_rk4_store", self.ctx.handle, N.dptr(out["xA"]), N.dptr(out["zetaA"]), N.dptr(out["xV"]),
               N.dptr(out["xQ"]) if nQ else None, N.dptr(out["ke"]), 0)
        return out

    def close(self) -> None:
        self.ctx.close()


class DistributedPanelVelocity:
    """BVERK4 over torch.distributed ranks with target sharding and a per-stage all-gather."""

    def __init__(self, device: int = 0, precision="fp32c", backend=None, group=None, comm=None):
        """comm: the collective layer (torch.distributed by default; any object with its
        get_rank / get_world_size / all_gather / all_reduce / barrier / ReduceOp)."""
        self._owns_group = False
        if comm is None:
            from datetime import timedelta

            import torch.distributed as comm

            if not comm.is_initialized():
                # a short timeout: a rank that dies makes the others' next collective fail
                comm.init_process_group("nccl", timeout=timedelta(seconds=180))
                self._owns_group = True
        dist = comm
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.backend = backend if backend is not None else LibBackend(device, precision)
        self.ranges: Ranges | None = None
        self._kes = []

    @property
    def ctx(self):
        return self.backend.ctx

    def bind_stream(self, stream) -> None:
        self.backend.bind_stream(stream)

    def barrier(self) -> None:
        self.dist.barrier(group=self.group)

    def max_over_ranks(self, value: float) -> float:
        t = self.backend.empty(1, 1)
        t.fill_(value)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX, group=self.group)
        return float(t.item())

    def load(self, w) -> None:
        """Every rank loads the full state (replicated data, as in the reference). The ranks
        first agree on the sizes: a rank whose arrays are short (or long) makes every rank raise
        ValueError here, before any stage exchange could wait on mismatched messages."""
        sizes = self.backend.empty(1, 3)
        sizes[0, 0], sizes[0, 1], sizes[0, 2] = float(w.nA), float(w.nV), float(w.nQ)
        seen = [self.backend.empty(1, 3) for _ in range(self.world)]
        self.dist.all_gather(seen, sizes, group=self.group)
        got = [tuple(int(v) for v in t.reshape(-1).tolist()) for t in seen]
        if any(g != got[0] for g in got):
            raise ValueError(f"ranks disagree on (nA, nV, nQ): {got}")
        self.w = w
        self.nA, self.nV, self.nQ = w.nA, w.nV, w.nQ
        self.ranges = Ranges(load_balance(w.nA, self.world), load_balance(w.nV, self.world),
                             load_balance(w.nQ, self.world))
        self.backend.load(w)
        # stage-1 sources of the first step; afterwards the exchanged source rows are the only
        # complete copy (a rank's own state arrays hold current values for its rows only)
        self.backend.pack_sources()
        self._kes = []

    @property
    def totalKE(self) -> list[float]:
        """Stage-1 kinetic energy of every step advanced since load() (sum over ranks)."""
        return [float(k.reshape(-1)[0].item()) for k in self._kes]

    def _allgather_rows(self, which: int, starts, ends, total: int) -> None:
        """Every rank exports its rows [start, end) of `which`; all ranks import all rows."""
        width = WIDTH[which]
        lens = ends - starts
        cap = int(lens.max()) if lens.size else 0
        if cap == 0:
            return
        send = self.backend.empty(cap, width)
        me = self.rank
        self.backend.export_rows(which, int(starts[me]), int(lens[me]), send)
        recv = [self.backend.empty(cap, width) for _ in range(self.world)]
        self.dist.all_gather(recv, send, group=self.group)
        for r in range(self.world):
            if r != me and lens[r] > 0:
                self.backend.import_rows(which, int(starts[r]), int(lens[r]), recv[r])

    def advance(self, dt: float, nsteps: int = 1) -> None:
        """nsteps RK4 steps of every rank's target rows, one source exchange per stage."""
        rng = self.ranges.rank(self.rank)
        for _ in range(nsteps):
            for s in range(4):
                self.backend.stage(s, dt, rng)
                if s == 0:
                    ke = self.backend.stage_ke().clone()
                    self.dist.all_reduce(ke, group=self.group)
                    self._kes.append(ke)
                # next stage's (or next step's) sources: everyone's active rows
                self._allgather_rows(SOURCES, *self.ranges.a, self.nA)

    def store(self) -> dict:
        """Gather the final state of every class to every rank (ScatterPanels needs all rows)."""
        self._allgather_rows(XA, *self.ranges.a, self.nA)
        self._allgather_rows(ZETA, *self.ranges.a, self.nA)
        self._allgather_rows(XV, *self.ranges.v, self.nV)
        if self.nQ:
            self._allgather_rows(XQ, *self.ranges.q, self.nQ)
        return self.backend.state()

    def close(self) -> None:
        self.backend.close()
        if self._owns_group:
            self.dist.destroy_process_group()
            self._owns_group = False
