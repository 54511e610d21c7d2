"""The target-sharded driver (dist.py) through torch.distributed's NCCL backend on one GPU: a
process group of world size 1 (the only size one GPU allows, since NCCL takes one rank per device)
runs the real all-gather of the packed source rows and the all-reduce of the kinetic energy on
the library's stream, in a child process so the test process keeps no process group. With one
rank every stage covers all rows, so the result must equal, bit for bit, the same steps through
the library's own tc_rk4_advance (the same kernels on the same data), and match the oracle."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
pytestmark = pytest.mark.gpu

CHILD = r"""
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from thesiscode_b200 import _native as N, configs
from thesiscode_b200.dist import DistributedPanelVelocity
from thesiscode_b200.panel_velocity import Context
prec = sys.argv[2]
w = configs.rh4(level=4, parity=True, dt=0.01)
drv = DistributedPanelVelocity(0, prec)
assert drv.world == 1 and drv.dist.get_backend() == "nccl"
drv.load(w)
drv.advance(w.dt, 2)
st = drv.store()
tke = drv.totalKE
drv.close()
ctx = Context(0, prec)
ctx.set_omega(w.omega)
ctx.set_deltas(*w.deltas)
N.call("tc_rk4_load", ctx.handle, N.dptr(w.xA), N.dptr(w.zetaA), N.dptr(w.areaA), w.nA, N.dptr(w.xV), w.nV,
       N.dptr(w.xQ), w.nQ, 0)
ke = np.zeros(2)
N.call("tc_rk4_advance", ctx.handle, w.dt, 2, N.dptr(ke))
xA, zA, xV, xQ = np.zeros_like(w.xA), np.zeros_like(w.zetaA), np.zeros_like(w.xV), np.zeros_like(w.xQ)
N.call("tc_rk4_store", ctx.handle, N.dptr(xA), N.dptr(zA), N.dptr(xV), N.dptr(xQ), None, 0)
ctx.close()
same = all(np.array_equal(a, b) for a, b in ((st["xA"], xA), (st["zetaA"], zA), (st["xV"], xV), (st["xQ"], xQ)))
np.savez(sys.argv[3], xA=st["xA"], zetaA=st["zetaA"], xV=st["xV"], xQ=st["xQ"], tke=np.array(tke), ke=ke)
print(json.dumps({"bitwise_equal_to_advance": bool(same)}))
"""


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32c", 3e-7)])
def test_nccl_world1_driver_equals_advance_and_oracle(gpu, tmp_path, precision, tol):
    from oracle import oracle as O
    from thesiscode_b200 import configs

    env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(free_port()), RANK="0", WORLD_SIZE="1",
               LOCAL_RANK="0", NCCL_NVLS_ENABLE="0")
    out = tmp_path / "state.npz"
    r = subprocess.run([sys.executable, "-c", CHILD, str(ROOT), precision, str(out)], capture_output=True,
                       text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-3000:]
    assert json.loads(r.stdout.strip().splitlines()[-1])["bitwise_equal_to_advance"]
    st = np.load(out)
    np.testing.assert_array_equal(st["tke"], st["ke"])
    w = configs.rh4(level=4, parity=True, dt=0.01)
    xV, xA, zA, xQ = w.xV, w.xA, w.zetaA, w.xQ
    for _ in range(2):
        xV, xA, zA, xQ, *_ = O.bve_rk4(xV, xA, zA, w.areaA, xQ, w.dt, w.omega, w.deltas,
                                      nthreads=os.cpu_count() or 1)
    assert np.abs(st["xA"] - xA).max() <= tol * np.abs(xA - w.xA).max()
    assert np.abs(st["xV"] - xV).max() <= tol * np.abs(xV - w.xV).max()
    assert np.abs(st["xQ"] - xQ).max() <= tol * np.abs(xQ - w.xQ).max()
    assert np.abs(st["zetaA"] - zA).max() <= tol * np.abs(zA - w.zetaA).max()
