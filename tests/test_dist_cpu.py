"""Multi-rank driver (thesiscode_b200.dist) on CPU: world sizes 2 and 3, gloo.

The driver's host logic - LoadBalance ranges (PanelVelocityParallel.f90:
167-213), one all-gather of the next stage's source rows per stage (the
reference's per-stage MPI_BCAST loops, :476-489), the final gather - runs
unchanged; the per-rank stage arithmetic comes from a test backend built on
the CPU oracle, which keeps the reference's rounding. Parallel results must
equal the serial oracle bit for bit, as the reference's MPI and serial
modules do. Failure detection is tested on the host: a rank that raises
before its first collective makes the other rank's collective fail within
the process-group timeout instead of hanging.
"""
import os
import socket
import sys
import traceback
from datetime import timedelta
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
SOURCES, XA, ZETA, XV, XQ, KE = range(6)


class OracleBackend:
    """Per-rank stage primitives with the library's semantics, computed by the CPU oracle.
    Source rows are (x, y, z, zeta) so the oracle rounds (cross*zeta)*area like the serial run."""

    ctx = None

    def __init__(self):
        import torch

        self.torch = torch

    def bind_stream(self, stream):
        pass

    def load(self, w):
        self.w = w
        self.x0A, self.z0 = w.xA.copy(), w.zetaA.copy()
        self.x0V, self.x0Q = w.xV.copy(), w.xQ.copy()
        self.xiV, self.xiQ = w.xV.copy(), w.xQ.copy()
        self.newA, self.newZ = np.zeros_like(self.x0A), np.zeros_like(self.z0)
        self.newV, self.newQ = np.zeros_like(self.x0V), np.zeros_like(self.x0Q)
        self.src = np.zeros((w.nA, 4))
        self.ke = np.zeros(w.nA)
        self.ke_t = self.torch.zeros(1, dtype=self.torch.float64)

    def pack_sources(self):
        self.src[:, :3] = self.x0A
        self.src[:, 3] = self.z0

    def stage(self, s, dt, rng):
        from oracle import oracle as O

        w = self.w
        a0, a1, v0, v1, q0, q1 = rng
        tV = self.x0V if s == 0 else self.xiV
        tQ = self.x0Q if s == 0 else self.xiQ
        dXA, dVA, dXV, dXQ = O.bve_stage(self.src[:, :3], self.src[:, 3], w.areaA, tV, tQ, w.omega,
                                         w.deltas, rng)
        if s == 0:
            acc = 0.0
            for j in range(a0, a1):
                u = dXA[j]
                k2 = u[0] * u[0]
                k2 = k2 + u[1] * u[1]
                k2 = k2 + u[2] * u[2]
                self.ke[j] = k2
                acc = acc + k2 * w.areaA[j]
            self.ke_t.fill_(0.5 * acc)
        div = 6.0 if s in (0, 3) else 3.0
        for (x0, new, xi, u, lo, hi) in ((self.x0A, self.newA, None, dXA, a0, a1),
                                         (self.x0V, self.newV, self.xiV, dXV, v0, v1),
                                         (self.x0Q, self.newQ, self.xiQ, dXQ, q0, q1)):
            k = dt * u[lo:hi]
            base = x0[lo:hi] if s == 0 else new[lo:hi]
            nv = base + k / div
            if s < 3:
                new[lo:hi] = nv
                nxt = x0[lo:hi] + (k if s == 2 else 0.5 * k)
                if xi is not None:
                    xi[lo:hi] = nxt
                else:
                    self.src[lo:hi, :3] = nxt
            else:
                x0[lo:hi] = nv
                if xi is None:
                    self.src[lo:hi, :3] = nv
        kz = dt * dVA[a0:a1]
        zbase = self.z0[a0:a1] if s == 0 else self.newZ[a0:a1]
        zn = zbase + kz / div
        if s < 3:
            self.newZ[a0:a1] = zn
            self.src[a0:a1, 3] = self.z0[a0:a1] + (kz if s == 2 else 0.5 * kz)
        else:
            self.z0[a0:a1] = zn
            self.src[a0:a1, 3] = zn

    def stage_ke(self):
        return self.ke_t

    def _buf(self, which):
        return {SOURCES: self.src, XA: self.x0A, ZETA: self.z0.reshape(-1, 1), XV: self.x0V,
                XQ: self.x0Q, KE: self.ke.reshape(-1, 1)}[which]

    def empty(self, rows, width):
        return self.torch.empty((rows, width), dtype=self.torch.float64)

    def export_rows(self, which, r0, n, out):
        out[:n] = self.torch.from_numpy(np.ascontiguousarray(self._buf(which)[r0:r0 + n]))

    def import_rows(self, which, r0, n, src):
        self._buf(which)[r0:r0 + n] = src[:n].numpy()

    def state(self):
        return dict(xA=self.x0A.copy(), zetaA=self.z0.copy(), xV=self.x0V.copy(), xQ=self.x0Q.copy(),
                    ke=self.ke.copy())

    def close(self):
        pass


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_dir, mode):
    sys.path.insert(0, str(ROOT))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch.distributed as dist

    from thesiscode_b200 import configs
    from thesiscode_b200.dist import DistributedPanelVelocity

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=10))
    try:
        if mode == "fail" and rank == 1:
            raise RuntimeError("injected failure on rank 1 before its first collective")
        w = configs.rh4(level=2, parity=True, dt=0.01)
        if mode == "short" and rank == 1:  # a rank whose active-panel arrays lost their last rows
            w.xA, w.zetaA, w.areaA = w.xA[:-7], w.zetaA[:-7], w.areaA[:-7]
        drv = DistributedPanelVelocity(backend=OracleBackend())
        drv.load(w)
        drv.advance(w.dt, 2)
        st = drv.store()
        np.savez(Path(out_dir) / f"rank{rank}.npz", tke=np.array(drv.totalKE), **st)
    except Exception as e:  # recorded for the parent test
        Path(out_dir, f"rank{rank}.err").write_text(f"{type(e).__name__}: {e}\n{traceback.format_exc()}")
    finally:
        try:
            if mode == "ok" or mode == "short":
                dist.destroy_process_group()
        except Exception:
            pass


def _spawn(mode, tmp_path, world=2):
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, str(tmp_path), mode)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    alive = [p for p in procs if p.is_alive()]
    for p in alive:
        p.kill()
    assert not alive, "a rank hung"


@pytest.mark.parametrize("world", [2, 3])
def test_ranks_match_serial_oracle_bitwise(tmp_path, native_built, world):
    """World size 3 gives ragged LoadBalance ranges (320 panels: 106, 106, 108 rows)."""
    from oracle import oracle as O
    from thesiscode_b200 import configs

    _spawn("ok", tmp_path, world=world)
    errs = list(tmp_path.glob("*.err"))
    assert not errs, errs[0].read_text()
    w = configs.rh4(level=2, parity=True, dt=0.01)
    xV, xA, zA, xQ = w.xV, w.xA, w.zetaA, w.xQ
    tkes = []
    for _ in range(2):
        xV, xA, zA, xQ, tke, ke, _ = O.bve_rk4(xV, xA, zA, w.areaA, xQ, w.dt, w.omega, w.deltas)
        tkes.append(tke)
    for r in range(world):
        g = np.load(tmp_path / f"rank{r}.npz")
        np.testing.assert_array_equal(g["xA"], xA)
        np.testing.assert_array_equal(g["zetaA"], zA)
        np.testing.assert_array_equal(g["xV"], xV)
        np.testing.assert_array_equal(g["xQ"], xQ)
        np.testing.assert_allclose(g["tke"], tkes, rtol=1e-14)


def test_failed_rank_surfaces_as_error_not_hang(tmp_path, native_built):
    _spawn("fail", tmp_path)
    e1 = (tmp_path / "rank1.err").read_text()
    assert "injected failure" in e1
    e0 = tmp_path / "rank0.err"
    assert e0.exists(), "rank 0 finished although its peer never joined the collective"


def test_short_buffer_on_one_rank_is_an_error_on_every_rank(tmp_path, native_built):
    _spawn("short", tmp_path)
    for r in range(2):
        e = tmp_path / f"rank{r}.err"
        assert e.exists(), f"rank {r} ran on with mismatched sizes"
        assert "ranks disagree on (nA, nV, nQ)" in e.read_text()
