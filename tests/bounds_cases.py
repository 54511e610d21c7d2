"""Cases that tests/test_bounds_check_gpu.py runs in a child process.

A child process can load either build of the library: the index-checked build
(TC_LIBRARY=checked) or the release build.

    python tests/bounds_cases.py results OUT.npz
        Runs a fixed set of calls and saves their results together with the
        device's index-check record. The parent compares the two builds bit
        for bit.
    python tests/bounds_cases.py caps OUT.json
        Checked build only. Runs each case once without a cap. It then caps one
        index-check site's declared extent below what the call touches, so that
        the check must fire. The arrays keep their real size, so every access
        that passes the check is still in bounds. It records what the device's
        record shows, removes the cap, and runs the case again.
"""
from __future__ import annotations

import ctypes
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

from thesiscode_b200 import _native as N  # noqa: E402
from thesiscode_b200 import configs  # noqa: E402
from thesiscode_b200.batch import batch_rk4  # noqa: E402
from thesiscode_b200.panel_velocity import Context  # noqa: E402

CAP = 7


def _ctx(prec, w):
    ctx = Context(0, prec)
    ctx.set_omega(w.omega)
    ctx.set_deltas(*w.deltas)
    return ctx


def _rh4():
    return configs.rh4(level=3, parity=True)  # 1,280 panels, 642 vertices, 420 divided panels


def _batch():
    ws = configs.batched_gaussians(count=6, seed=4, levels=(1, 2, 3))
    ws[2].xV = np.zeros((0, 3))
    return ws


def velocity_vertex(ctx, w):
    return ctx.velocity(N.TC_VERTEX, w.xV, w.xA, w.zetaA, w.areaA)[0]


def rk4_step(ctx, w, nsteps=1):
    s = w.copy()
    tke, ke = ctx.rk4_step(s.xA, s.zetaA, s.areaA, s.xV, s.xQ, 0.01, nsteps=nsteps)
    return np.concatenate([s.xA.ravel(), s.zetaA, s.xV.ravel(), s.xQ.ravel(), tke, ke])


def batch(ctx, ws):
    ws = [w.copy() for w in ws]
    tke = batch_rk4(ctx, ws, 0.01, 2, graph=False, autotune=False)
    return np.concatenate([np.concatenate([w.xA.ravel(), w.zetaA, w.xV.ravel()]) for w in ws]
                          + [np.asarray(tke).ravel()])


def noalloc(ctx, w):
    import torch

    dev = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (w.xV, w.xA, w.zetaA, w.areaA)]
    u = torch.zeros((w.nV, 3), dtype=torch.float64, device="cuda")
    p = [ctypes.c_void_p(t.data_ptr()) for t in dev + [u]]
    N.call("tc_bs_velocity_device_noalloc", ctx.handle, N.TC_VERTEX, p[0], w.nV, p[1], p[2], p[3],
           w.nA, 0, w.nV, p[4], None)
    torch.cuda.synchronize()
    return u.cpu().numpy()


def strat(ctx, w):
    s = w.copy()
    relA, _, tke, ke = ctx.strat_rk4_step(s.xA, w.meta["absVortA"], s.areaA, s.xV, s.xQ,
                                          w.meta["t0"], w.dt, 1)
    return np.concatenate([s.xA.ravel(), relA, s.xV.ravel(), tke, ke])


def adjoint(ctx, w, steps=3):
    J, gz, gx = np.zeros(1), np.zeros(w.nA), np.zeros((w.nA, 3))
    N.call("tc_rk4_adjoint", ctx.handle, N.dptr(w.xA), N.dptr(w.zetaA), N.dptr(w.areaA), w.nA, 0.01,
           steps, 2, N.TC_J_ENSTROPHY, 0, N.dptr(J), N.dptr(gz), N.dptr(gx))
    return np.concatenate([J, gz, gx.ravel()])


def results(out_path):
    w, ws = _rh4(), _batch()
    st = configs.stratosphere(level=3)
    out = {}
    for prec in ("fp64", "fp32c"):
        ctx = _ctx(prec, w)
        u, v = ctx.velocity(N.TC_ACTIVE, None, w.xA, w.zetaA, w.areaA, 100, 1100)
        out[f"{prec}_active_u"], out[f"{prec}_active_v"] = u, v
        out[f"{prec}_vertex_u"] = velocity_vertex(ctx, w)
        out[f"{prec}_passive_u"] = ctx.velocity(N.TC_PASSIVE, w.xQ, w.xA, w.zetaA, w.areaA)[0]
        out[f"{prec}_rk4"] = rk4_step(ctx, w, nsteps=3)  # steps 2-3 replay a CUDA graph
        out[f"{prec}_noalloc"] = noalloc(ctx, w)
        if prec == "fp64":
            out["fp64_adjoint"] = adjoint(ctx, w)
        ctx.close()
        ctx = _ctx(prec, st)
        s = st.copy()
        relA, _, tke, ke = ctx.strat_rk4_step(s.xA, st.meta["absVortA"], s.areaA, s.xV, s.xQ,
                                              st.meta["t0"], st.dt, nsteps=2)
        out[f"{prec}_strat"] = np.concatenate([s.xA.ravel(), relA, s.xV.ravel(), tke, ke])
        ctx.close()
        ctx = _ctx(prec, ws[0])
        out[f"{prec}_batch"] = batch(ctx, ws)
        ctx.close()
    rec = N.bounds_status(0, reset=True)
    out["record"] = np.array([rec["count"], rec["site"], rec["index"], rec["extent"]])
    out["checked"] = np.array(N.lib().tc_bounds_checked())
    np.savez(out_path, **out)


# (site, precision, case): each case touches its site on every call
CAP_CASES = [
    ("PAIR_X", "fp32c", "velocity"), ("PAIR_PERM", "fp32c", "velocity"),
    ("PAIR_SRC", "fp32c", "velocity"), ("PAIR_OUT", "fp32c", "velocity"),
    ("PAIR_X", "fp64", "velocity"), ("PAIR_SRC", "fp64", "velocity"),
    ("PAIR_OUT", "fp64", "velocity"),
    ("PACK_IN", "fp32c", "velocity"), ("PACK_OUT", "fp32c", "velocity"),
    ("EPI_PERM", "fp32c", "velocity"), ("EPI_X", "fp32c", "velocity"),
    ("EPI_PARTIAL", "fp32c", "velocity"), ("EPI_OUT", "fp32c", "velocity"),
    ("EPI_PARTIAL", "fp32c", "noalloc"),
    ("STAGE_PERM", "fp32c", "rk4"), ("STAGE_STATE", "fp32c", "rk4"),
    ("STAGE_PARTIAL", "fp32c", "rk4"), ("STAGE_ACTIVE", "fp32c", "rk4"),
    ("STAGE_KEBLOCK", "fp32c", "rk4"), ("STAGE_STATE", "fp64", "rk4"),
    ("BATCH_SEG", "fp32c", "batch"), ("BATCH_SEG", "fp64", "batch"),
    ("STAGE_CHUNKS", "fp32c", "batch"),
    ("ADJ_ROW_IN", "fp64", "adjoint"), ("ADJ_ROW_OUT", "fp64", "adjoint"),
    ("ADJ_COMBINE", "fp64", "adjoint"),
    ("ORDER_X", "fp32c", "velocity"), ("ORDER_KEYS", "fp32c", "velocity"),
    ("ORDER_X", "fp32c", "rk4"), ("ORDER_KEYS", "fp32c", "noalloc"),
    ("ORDER_X", "fp32c", "batch"), ("ORDER_KEYS", "fp32c", "batch"), ("BATCH_KE", "fp64", "batch"),
    ("PACK_IN", "fp64", "strat"), ("PACK_OUT", "fp64", "strat"),
]
SITE_IDS = {name: i for i, name in enumerate(
    ["", "PAIR_X", "PAIR_PERM", "PAIR_SRC", "PAIR_OUT", "BATCH_SEG", "PACK_IN", "PACK_OUT",
     "EPI_PERM", "EPI_X", "EPI_PARTIAL", "EPI_OUT", "STAGE_PERM", "STAGE_STATE",
     "STAGE_PARTIAL", "STAGE_CHUNKS", "STAGE_ACTIVE", "STAGE_KEBLOCK", "ADJ_ROW_IN",
     "ADJ_ROW_OUT", "ADJ_COMBINE", "ORDER_X", "ORDER_KEYS", "BATCH_KE"])}


def caps(out_path):
    w, ws = _rh4(), _batch()
    st = configs.stratosphere(level=3)
    runs = {"strat": lambda c: strat(c, st),"velocity": lambda c: velocity_vertex(c, w), "rk4": lambda c: rk4_step(c, w),
            "batch": lambda c: batch(c, ws), "noalloc": lambda c: noalloc(c, w),
            "adjoint": lambda c: adjoint(c, w)}
    report = []
    for site, prec, case in CAP_CASES:
        ctx = _ctx(prec, ws[0] if case == "batch" else st if case == "strat" else w)
        run = runs[case]
        base = run(ctx)
        clean_before = N.bounds_status(0, reset=True)["count"]
        N.call("tc_bounds_cap", ctx.handle, SITE_IDS[site], CAP)
        try:
            run(ctx)
            status = 0
        except N.TcError as e:  # a capped call may end in a non-finite result or a short read
            status = e.status
        rec = N.bounds_status(0, reset=True)
        N.call("tc_bounds_cap", ctx.handle, 0, -1)
        again = run(ctx)
        clean_after = N.bounds_status(0, reset=True)["count"]
        ctx.close()
        report.append(dict(site=site, site_id=SITE_IDS[site], precision=prec, case=case, cap=CAP,
                           clean_before=clean_before, status=status, record=rec,
                           clean_after=clean_after, same_after=bool(np.array_equal(base, again))))
    Path(out_path).write_text(json.dumps(report, indent=1))


if __name__ == "__main__":
    {"results": results, "caps": caps}[sys.argv[1]](sys.argv[2])
