#!/usr/bin/env python
"""Benchmark of the direct spherical Biot-Savart RK4 step on B200.

Metric: Biot-Savart interactions/s (one interaction = one (target, source)
pair evaluated; one RK4 step = 4 stages x [nA(nA-1) + (nV + nQ) nA]).

Default workload: Rossby-Haurwitz wave 4 (omega = K = Omega/14), icosahedral
level 8 (1,310,720 active panels + 655,362 vertices, about 1.97M targets),
delta = 0.005 for all targets, one RK4 step per timed step, FP32-compensated
pair arithmetic (the FP64 path is measured beside it). The Gaussian vortex at
level 7 (327,680 panels + 163,842 vertices, delta 0.01) is measured beside it
under the key "gaussian_l7".

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                    [--config rh4_l8|gaussian_l7|rh4_l4|jet_l6] [--precision fp32c|fp64]

Timing: CUDA events on the library's stream around each step, L2 flushed
(a 256 MiB write) between timed steps, max over ranks. The reference arm
(--impl reference) and the CPU baseline time the CPU FP64 restatement of the
reference loops (oracle/) in its timing build (compiled with the freedoms of
the reference's ifort -O2: vectorized, reassociated, reciprocal division) on
all host cores over a seeded sample of target rows, on inputs built from the
oracle's own restatement of the icosahedral grid generator (the reference arm
loads no part of the product library); errors are measured against the
strict parity build.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

FLOPS_PER_INTERACTION = 22  # dot 5, denominator 1, weight 1, cross 9, accumulate 6
L2_FLUSH_BYTES = 256 << 20
ERROR_ROWS_MAX = 24576  # rows of the strict-oracle error sample (a seeded subset)
# DRAM bytes (read + write) of one FP32C pair launch (the stage-1 launch of one RK4 step, every
# target class against all sources), from ncu captures (dram__bytes_read.sum +
# dram__bytes_write.sum) summarised in profiles/
PAIR_FP32C_DRAM_BYTES = {"rh4_l8": 328.61e6 + 204.19e6, "gaussian_l7": 28.02e6 + 52.43e6}


def build_workload(name: str, grid_source=None):
    """The named workload; grid_source (a callable level -> (xV, xA, areaA, xQ)) replaces the
    library's grid generator."""
    from thesiscode_b200 import configs

    if name == "gaussian_l7":
        return configs.gaussian(level=7, delta=0.01, dt=0.01, steps=1, grid_source=grid_source)
    if name == "rh4_l8":
        return configs.rh4(level=8, delta=0.005, dt=0.01, steps=1, grid_source=grid_source)
    if name == "rh4_l4":
        return configs.rh4(level=4, delta=0.0, dt=0.01, steps=10, grid_source=grid_source)
    if name == "jet_l6":
        return configs.jet(level=6, delta=0.02, dt=0.005, steps=20, grid_source=grid_source)
    raise SystemExit(f"unknown config {name}")


def oracle_workload(name: str, check=None):
    """The named workload on the oracle's icosahedral grid (oracle/icos_oracle.c); with `check`
    (the same workload from the library's generator) the two must agree bit for bit."""
    from oracle import oracle as O

    w = build_workload(name, grid_source=O.gathered_grid)
    if check is not None:
        for a, b in ((w.xA, check.xA), (w.zetaA, check.zetaA), (w.areaA, check.areaA), (w.xV, check.xV),
                     (w.xQ, check.xQ)):
            if not np.array_equal(a, b):
                raise SystemExit("the library's grid differs from the oracle's: inputs are not the same")
    return w


def workload_config(w, precision, scaling_note):
    return {"workload": f"{w.name}: {w.meta.get('ic', '')}", "level": w.level, "n_active": w.nA,
            "n_vertex": w.nV, "n_passive": w.nQ, "delta": w.deltas[0], "omega": w.omega, "dt": w.dt,
            "rk4_steps_per_step": 1, "arith": precision, "interactions_per_step": w.interactions_per_step(),
            "l2": "flushed between timed steps (256 MiB write)", "parallelism": scaling_note}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks(device: int) -> dict:
    from thesiscode_b200 import _native as N

    out = {}  # ffma, dfma: FMA/s; rcp32: MUFU reciprocals/s; far_pairs: pairs/s
    for key, kind, iters in (("ffma", N.TC_PROBE_FFMA, 65536), ("dfma", N.TC_PROBE_DFMA, 32768),
                             ("rcp32", N.TC_PROBE_RCP32, 16384),
                             ("far_pairs", N.TC_PROBE_FAR_PAIRS, 2048)):
        best = 0.0
        for _ in range(3):
            v = ctypes.c_double()
            N.call("tc_probe_peak", device, kind, iters, ctypes.byref(v))
            best = max(best, v.value)
        out[key] = best  # FMA/s
    return out


def stats(ctx, reset=False):
    from thesiscode_b200 import _native as N

    L, PL, PI = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
    ms = ctypes.c_double()
    N.call("tc_stats", ctx.handle, int(reset), ctypes.byref(L), ctypes.byref(PL), ctypes.byref(PI),
           ctypes.byref(ms))
    return L.value, PL.value, PI.value, ms.value


def time_device_steps(w, precision, steps, warmup, device, dist_driver=None):
    """Device-resident timing: state loaded once, `steps` RK4 steps timed one by one."""
    import torch

    from thesiscode_b200 import _native as N
    from thesiscode_b200.panel_velocity import Context

    stream = torch.cuda.Stream(device)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=f"cuda:{device}")
    if dist_driver is None:
        ctx = Context(device, precision)
        ctx.set_stream(stream.cuda_stream)
        ctx.set_omega(w.omega)
        ctx.set_deltas(*w.deltas)
        N.call("tc_rk4_load", ctx.handle, N.dptr(w.xA), N.dptr(w.zetaA), N.dptr(w.areaA), w.nA,
               N.dptr(w.xV), w.nV, N.dptr(w.xQ) if w.nQ else None, w.nQ, 0)

        def one_step():
            N.call("tc_rk4_advance", ctx.handle, w.dt, 1, None)
    else:
        ctx = dist_driver.ctx
        dist_driver.bind_stream(stream)
        dist_driver.load(w)

        def one_step():
            dist_driver.advance(w.dt, 1)

    with torch.cuda.stream(stream):
        for _ in range(warmup):
            one_step()
        torch.cuda.synchronize(device)
        N.call("tc_stats_enable_timing", ctx.handle, 1)
        stats(ctx, reset=True)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(steps)]
        if dist_driver is not None:
            dist_driver.barrier()
        torch.cuda.synchronize(device)
        clocks = ClockSampler(device)
        clocks.start()
        t_wall = time.perf_counter()
        for k in range(steps):
            flush.fill_(float(k))
            ev[k][0].record(stream)
            one_step()
            ev[k][1].record(stream)
        torch.cuda.synchronize(device)
        t_wall = time.perf_counter() - t_wall
        if dist_driver is not None:
            dist_driver.barrier()
        clk = clocks.stop()
        N.call("tc_stats_enable_timing", ctx.handle, 0)
        step_ms = [a.elapsed_time(b) for a, b in ev]
        launches, pair_launches, pair_inter, pair_ms = stats(ctx, reset=True)
    return dict(step_ms=step_ms, total_ms=sum(step_ms), wall_s=t_wall, launches=launches,
                pair_launches=pair_launches, pair_interactions=pair_inter, pair_ms=pair_ms,
                clocks=clk, ctx=ctx)


def time_e2e(w, precision, steps, device):
    """End to end through the public host-pointer call tc_rk4_step: pinned host inputs copied
    in, one fused RK4 step, results (positions, vorticity, kinetic energy) copied out."""
    import torch

    from thesiscode_b200 import _native as N
    from thesiscode_b200.panel_velocity import Context

    ctx = Context(device, precision)
    stream = torch.cuda.Stream(device)
    ctx.set_stream(stream.cuda_stream)
    ctx.set_omega(w.omega)
    ctx.set_deltas(*w.deltas)

    def pinned(a):
        t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
        t.numpy()[...] = a
        return t

    xA, zA, aA, xV = pinned(w.xA), pinned(w.zetaA), pinned(w.areaA), pinned(w.xV)
    xQ = pinned(w.xQ if w.nQ else np.zeros((0, 3)))
    ke = pinned(np.zeros(w.nA))
    tke = np.zeros(1)

    def call():
        N.call("tc_rk4_step", ctx.handle, *(ctypes.cast(t.data_ptr(), N.dp) for t in (xA, zA, aA)),
               w.nA, ctypes.cast(xV.data_ptr(), N.dp), w.nV,
               ctypes.cast(xQ.data_ptr(), N.dp) if w.nQ else None, w.nQ, w.dt, 1, N.dptr(tke),
               ctypes.cast(ke.data_ptr(), N.dp))

    call()  # warm-up (allocations)
    times = []
    for _ in range(steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        call()
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    ctx.close()
    D = 8
    h2d = (3 * w.nA + 2 * w.nA + 3 * w.nV + 3 * w.nQ) * D
    d2h = (3 * w.nA + w.nA + 3 * w.nV + 3 * w.nQ + w.nA + 1) * D
    return dict(ms=sum(times) / len(times), h2d=h2d, d2h=d2h)


def time_e2e_dist(w, driver, steps):
    """End to end at N ranks through the distributed driver's public calls: every rank loads the
    host arrays (H2D), advances one RK4 step (its target rows, one source all-gather per stage)
    and stores the full state back to host arrays (all-gather + D2H). CUDA events on the
    driver's stream per rank, median over steps, max over ranks."""
    import torch

    stream = torch.cuda.Stream()
    driver.bind_stream(stream)
    times = []
    for _ in range(steps + 1):  # the first call allocates
        driver.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            driver.load(w)
            driver.advance(w.dt, 1)
            driver.store()
            e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    ms = driver.max_over_ranks(statistics.median(times[1:]))
    D = 8
    h2d = (3 * w.nA + 2 * w.nA + 3 * w.nV + 3 * w.nQ) * D * driver.world
    d2h = (3 * w.nA + w.nA + 3 * w.nV + 3 * w.nQ + w.nA) * D * driver.world
    return dict(ms=ms, h2d=h2d, d2h=d2h)


def time_adjoint(device, level=6, steps=20, ckpt=5):
    """Adjoint/forward time ratio on the zonal-jet workload (level 6, delta 0.02, dt 0.005, FP64,
    J = sum zeta^2 A). The adjoint's phases are CUDA-event timed inside the library (forward sweep
    with checkpoints, recomputation of checkpoint segments, backward sweep); the forward reference
    is the same steps through tc_rk4_advance on device-resident state."""
    import torch

    from thesiscode_b200 import _native as N
    from thesiscode_b200.panel_velocity import Context

    w = build_workload("jet_l6")
    ctx = Context(device, "fp64")
    stream = torch.cuda.Stream(device)
    ctx.set_stream(stream.cuda_stream)
    ctx.set_omega(w.omega)
    ctx.set_deltas(*w.deltas)
    J, gz, gx = np.zeros(1), np.zeros(w.nA), np.zeros((w.nA, 3))
    out = {"workload": f"jet level {w.level} ({w.nA} panels), delta 0.02, {steps} RK4 steps dt {w.dt}, "
                       "J = sum zeta^2 A, FP64"}

    def fwd_ms():
        N.call("tc_rk4_load", ctx.handle, N.dptr(w.xA), N.dptr(w.zetaA), N.dptr(w.areaA), w.nA, None, 0,
               None, 0, 0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        N.call("tc_rk4_advance", ctx.handle, w.dt, steps, None)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1)

    fwd_ms()
    tf = min(fwd_ms() for _ in range(2))
    out["forward_ms"] = tf
    for name, ck in (("checkpoint_every_5", ckpt), ("stage_inputs_kept", steps)):
        ph = np.zeros(3)
        for _ in range(2):
            N.call("tc_rk4_adjoint", ctx.handle, N.dptr(w.xA), N.dptr(w.zetaA), N.dptr(w.areaA), w.nA, w.dt,
                   steps, ck, N.TC_J_ENSTROPHY, 0, N.dptr(J), N.dptr(gz), N.dptr(gx))
        N.call("tc_adjoint_phase_ms", ctx.handle, N.dptr(ph))
        out[name] = {"checkpoint_every": ck, "forward_sweep_ms": ph[0], "recompute_ms": ph[1],
                     "backward_ms": ph[2],
                     "adjoint_over_forward": (ph[1] + ph[2]) / tf,
                     "gradient_over_forward": (ph[0] + ph[1] + ph[2]) / tf}
    out["J"] = float(J[0])
    ctx.close()
    return out


def time_batch(device, steps=10):
    """Batched ensemble: 64 Gaussian vortices (seed 4), levels 3-6, 10 RK4 steps each, FP32C,
    one CUDA-graph launch per call. The first call autotunes and captures; the second is timed
    end to end (host arrays in and out)."""
    from thesiscode_b200 import configs
    from thesiscode_b200.batch import batch_info, batch_rk4
    from thesiscode_b200.panel_velocity import Context

    ws = configs.batched_gaussians(count=64, seed=4, levels=(3, 4, 5, 6))
    ctx = Context(device, "fp32c")
    ctx.set_omega(ws[0].omega)
    ctx.set_deltas(*ws[0].deltas)
    t = time.perf_counter()
    batch_rk4(ctx, [w.copy() for w in ws], ws[0].dt, steps)
    first = time.perf_counter() - t
    t = time.perf_counter()
    batch_rk4(ctx, ws, ws[0].dt, steps)
    dt = time.perf_counter() - t
    info = batch_info(ctx)
    ctx.close()
    inter = steps * sum(w.interactions_per_step() for w in ws)
    return {"workload": "64 Gaussian vortices (seed 4), icosahedral levels 3-6, beta in [4,20], "
                        f"{steps} RK4 steps each, FP32C, one CUDA graph", "interactions": inter,
            "seconds": dt, "value": inter / dt, "unit": "interactions/s",
            "first_call_seconds": first,
            "levels": sorted(set(w.level for w in ws)), "autotuned": info}


def sample_rows(w, frac, seed=11):
    rng = np.random.default_rng(seed)
    ra = np.sort(rng.choice(w.nA, max(1, int(w.nA * frac)), replace=False)).astype(np.int32)
    rv = np.sort(rng.choice(w.nV, max(1, int(w.nV * frac)), replace=False)).astype(np.int32)
    return ra, rv


def sample_frac(w, seconds, threads, lo=1.0 / 64):
    """Fraction of target rows (a power of two) that the CPU oracle sums in about `seconds`
    on `threads` host threads, from a timed 1/256 sample; at least `lo`, at most all rows."""
    cal = cpu_baseline(w, frac=1.0 / 256, threads=threads)["seconds"]
    want = seconds / max(cal, 1e-6) / 256
    frac = lo
    while frac * 2 <= min(want, 1.0):
        frac *= 2
    return frac


def cpu_baseline(w, frac=1.0 / 64, threads=None):
    """The reference's loops restated in C (oracle/), in the timing build that matches the
    reference's own compiler settings (ifort -O2: vectorized, reassociation, reciprocal
    division, contraction; the host's highest x86-64 level), on all host cores over a seeded
    sample (`frac` of the target rows) of one RK4 stage; returns interactions/s."""
    from oracle import oracle as O

    threads = threads or os.cpu_count() or 1
    level = O.fast_lib()[1]
    ra, rv = sample_rows(w, frac)
    t = time.perf_counter()
    O.rows(0, ra, None, w.xA, w.zetaA, w.areaA, delta=w.deltas[0], nthreads=threads, fast=True)
    O.rows(1, rv, w.xV, w.xA, w.zetaA, w.areaA, delta=w.deltas[1], nthreads=threads, fast=True)
    dt = time.perf_counter() - t
    inter = ra.size * (w.nA - 1) + rv.size * w.nA
    return dict(value=inter / dt, seconds=dt, cores=threads, rows=(ra, rv), isa=level,
                build=f"oracle C port, gcc -O3 -fassociative-math -freciprocal-math "
                      f"-ffp-contract=fast, x86-64-{level} (the reference builds with ifort -O2)",
                sample=f"one RK4 stage, seeded 1/{round(1 / frac)} of target rows "
                       f"({ra.size} active + {rv.size} vertex rows x {w.nA} sources)")


def oracle_sums(w, rows, threads):
    """The strict (parity) oracle's sums on the sampled rows of stage 1."""
    from oracle import oracle as O

    ra, rv = rows
    return (O.rows(0, ra, None, w.xA, w.zetaA, w.areaA, delta=w.deltas[0], nthreads=threads),
            O.rows(1, rv, w.xV, w.xA, w.zetaA, w.areaA, delta=w.deltas[1], nthreads=threads))


def gpu_stage1_errors(w, precision, device, rows, sums):
    """Max/RMS of |u_gpu - u_oracle| / max|u_oracle| on the sampled rows of stage 1."""
    from thesiscode_b200 import _native as N
    from thesiscode_b200.panel_velocity import Context

    ctx = Context(device, precision)
    ctx.set_omega(w.omega)
    ctx.set_deltas(*w.deltas)
    dA, _ = ctx.velocity(N.TC_ACTIVE, None, w.xA, w.zetaA, w.areaA)
    dV, _ = ctx.velocity(N.TC_VERTEX, w.xV, w.xA, w.zetaA, w.areaA)
    ctx.close()
    ra, rv = rows
    diff = np.concatenate([dA[ra] - sums[0], dV[rv] - sums[1]])
    ref = np.concatenate([sums[0], sums[1]])
    scale = np.abs(ref).max()
    return dict(max=float(np.abs(diff).max() / scale),
                rms=float(np.sqrt((diff ** 2).sum(1).mean()) / scale))


def error_sample(w, device, threads, max_rows=ERROR_ROWS_MAX):
    """Stage-1 velocity errors of both GPU paths against the strict parity oracle on a seeded
    sample of at most `max_rows` target rows (at most 1/8 of the rows)."""
    frac = min(1.0 / 8, max_rows / (w.nA + w.nV))
    err_rows = sample_rows(w, frac, seed=12)
    sums = oracle_sums(w, err_rows, threads)
    out = {p: gpu_stage1_errors(w, p, device, err_rows, sums) for p in ("fp32c", "fp64")}
    out["rows"] = int(err_rows[0].size + err_rows[1].size)
    return out


def time_side_workload(name, device, no_cpu, steps=3):
    """A second workload measured beside the headline: FP32C and FP64 device-resident step rates,
    their ratio and (unless no_cpu) the errors against the strict oracle."""
    w = build_workload(name)
    out = {"workload": workload_config(w, "fp32c", "1 GPU")["workload"], "level": w.level,
           "interactions_per_step": w.interactions_per_step()}
    for prec in ("fp32c", "fp64"):
        r = time_device_steps(w, prec, steps, 1, device)
        r["ctx"].close()
        out[prec] = {"value": w.interactions_per_step() * steps / (r["total_ms"] * 1e-3),
                     "ms_per_step": r["total_ms"] / steps,
                     "pair_ms_per_launch": r["pair_ms"] / max(r["pair_launches"], 1)}
    out["fp32c_over_fp64"] = out["fp32c"]["value"] / out["fp64"]["value"]
    if not no_cpu:
        out["error_vs_fp64_oracle"] = error_sample(oracle_workload(name, check=w), device,
                                                   os.cpu_count() or 1, max_rows=8192)
    return out


def time_config1(device, check=True, reps=5):
    """Config 1: Rossby-Haurwitz wave 4, level 4 (5,120 panels + 2,562 vertices), FP64, delta 0,
    ten RK4 steps of dt 0.01 per call, device-resident (tc_rk4_load once, tc_rk4_advance(10) timed
    by CUDA events, best of `reps`), and the displacement error of the ten steps against ten
    oracle BVERK4 steps."""
    import torch

    from oracle import oracle as O
    from thesiscode_b200 import _native as N
    from thesiscode_b200.panel_velocity import Context

    w = build_workload("rh4_l4")
    ctx = Context(device, "fp64")
    stream = torch.cuda.Stream(device)
    ctx.set_stream(stream.cuda_stream)
    ctx.set_omega(w.omega)
    ctx.set_deltas(*w.deltas)
    best = float("inf")
    for _ in range(reps + 1):  # the first call sizes buffers and captures the step graph
        N.call("tc_rk4_load", ctx.handle, N.dptr(w.xA), N.dptr(w.zetaA), N.dptr(w.areaA), w.nA, N.dptr(w.xV),
               w.nV, None, 0, 0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        N.call("tc_rk4_advance", ctx.handle, w.dt, w.steps, None)
        e1.record(stream)
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    xA, xV = np.zeros_like(w.xA), np.zeros_like(w.xV)
    N.call("tc_rk4_store", ctx.handle, N.dptr(xA), None, N.dptr(xV), None, None, 0)
    ctx.close()
    out = {"workload": f"{w.name}: {w.meta['ic']}, FP64, delta 0, {w.steps} RK4 steps of dt {w.dt}",
           "value": w.interactions_per_step() * w.steps / (best * 1e-3), "unit": "interactions/s",
           "ms_per_step": best / w.steps}
    if check:
        rV, rA, rz = w.xV, w.xA, w.zetaA
        for _ in range(w.steps):
            rV, rA, rz, *_ = O.bve_rk4(rV, rA, rz, w.areaA, np.zeros((0, 3)), w.dt, w.omega, w.deltas,
                                       nthreads=os.cpu_count() or 1)
        out["displacement_error_vs_fp64_oracle"] = float(max(
            np.abs(xA - rA).max() / np.abs(rA - w.xA).max(), np.abs(xV - rV).max() / np.abs(rV - w.xV).max()))
    return out


def run_ours(args):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    device = local
    torch.cuda.set_device(device)
    from thesiscode_b200 import _native as N

    N.lib()
    w = build_workload(args.config)
    driver = None
    if world > 1:
        from thesiscode_b200.dist import DistributedPanelVelocity

        driver = DistributedPanelVelocity(device, args.precision)
    peaks = measured_peaks(device)
    main = time_device_steps(w, args.precision, args.steps, args.warmup, device, driver)
    total_ms = main["total_ms"]
    if driver is not None:
        total_ms = driver.max_over_ranks(total_ms)
    value = w.interactions_per_step() * args.steps / (total_ms * 1e-3)
    fp_peak = (peaks["ffma"] if args.precision == "fp32c" else peaks["dfma"]) * 2.0
    pair_flops = FLOPS_PER_INTERACTION * main["pair_interactions"] / max(main["pair_launches"], 1)
    pair_ms_launch = main["pair_ms"] / max(main["pair_launches"], 1)
    achieved = pair_flops / (pair_ms_launch * 1e-3)
    line = {
        "metric": "Biot-Savart interactions/s (one RK4 step of the direct spherical sum)",
        "value": value, "unit": "interactions/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "strong" if world > 1 else "weak", "vs_baseline": None,
        "dtype": "f32 pairs (compensated, f64 accumulation)" if args.precision == "fp32c" else "f64",
        "data": "synthetic: analytic vorticity on a generated icosahedral grid (seeded)",
        "config": workload_config(w, args.precision, f"target-sharded x{world}" if world > 1 else "1 GPU"),
        "roofline": {"bound": "fp32" if args.precision == "fp32c" else "fp64",
                     "achieved": achieved / 1e12, "peak": fp_peak / 1e12, "unit": "TFLOP/s",
                     "frac": achieved / fp_peak,
                     "traffic": (PAIR_FP32C_DRAM_BYTES.get(args.config) if args.precision == "fp32c"
                                 else None),
                     "kernel": f"pair_{args.precision}_kernel",
                     "flops_per_interaction": FLOPS_PER_INTERACTION,
                     "pair_ms_per_launch": pair_ms_launch,
                     "peak_source": "measured live: CUDA-core FMA probe (tc_probe_peak) x 2 flops"},
        # FP32C executes one MUFU reciprocal per interaction (the XU pipe, 16 lanes per SM) beside
        # 7-11 FP32 operations: the hardware bound of the pair kernel, next to the 22-flop count
        "pipe_roofline": ({"pipe": "xu (MUFU rcp.approx.f32, one per interaction)",
                           "achieved": main["pair_interactions"] / max(main["pair_ms"] * 1e-3, 1e-30),
                           "peak": peaks["rcp32"], "unit": "reciprocals/s",
                           "frac": main["pair_interactions"] / max(main["pair_ms"] * 1e-3, 1e-30) / peaks["rcp32"],
                           "peak_source": "measured live: MUFU reciprocal probe (tc_probe_peak)",
                           # the kernel's own far-form step alone over a resident shared-memory
                           # tile (no staging, far tests, flushes or near tiles): the ceiling of
                           # the pair loop's instruction mix
                           "pair_loop_ceiling": {
                               "value": peaks["far_pairs"], "unit": "pairs/s",
                               "frac": main["pair_interactions"] / max(main["pair_ms"] * 1e-3, 1e-30)
                               / peaks["far_pairs"],
                               "source": "measured live: tc_probe_peak TC_PROBE_FAR_PAIRS"}}
                          if args.precision == "fp32c" else None),
        "gpu_launches": main["launches"],
        "gpu_launches_note": "the library's own kernels (pack, Hilbert keys, pair, stage epilogue, KE finalize); "
                             "each FP32C step also runs two CUB radix sorts (6 kernels each on this "
                             "toolkit: histogram, exclusive sum, 4 onesweep passes)",
        "clocks": main["clocks"],
    }
    e2e_dist = None
    if world > 1 and not args.quick:  # every rank takes part (collectives)
        e2e_dist = time_e2e_dist(w, driver, max(2, min(args.steps, 4)))
    if rank == 0:
        if e2e_dist is not None:
            line["e2e"] = {"value": w.interactions_per_step() / (e2e_dist["ms"] * 1e-3), "unit": "interactions/s",
                           "h2d_bytes_per_step": e2e_dist["h2d"], "d2h_bytes_per_step": e2e_dist["d2h"],
                           "ms_per_step": e2e_dist["ms"],
                           "api": f"DistributedPanelVelocity load/advance/store on {world} ranks (host arrays; "
                                  "bytes summed over ranks)"}
        if world == 1 and not args.quick:
            other = "fp64" if args.precision == "fp32c" else "fp32c"
            o = time_device_steps(w, other, max(1, min(args.steps, 3)), 1, device)
            o["ctx"].close()
            line[other] = {"value": w.interactions_per_step() * len(o["step_ms"]) / (o["total_ms"] * 1e-3),
                           "ms_per_step": o["total_ms"] / len(o["step_ms"])}
            fast = line["value"] if args.precision == "fp32c" else line[other]["value"]
            slow = line[other]["value"] if args.precision == "fp32c" else line["value"]
            line["fp32c_over_fp64"] = fast / slow
        if world == 1 and not args.quick:
            e2e = time_e2e(w, args.precision, max(2, min(args.steps, 4)), device)
            line["e2e"] = {"value": w.interactions_per_step() / (e2e["ms"] * 1e-3), "unit": "interactions/s",
                           "h2d_bytes_per_step": e2e["h2d"], "d2h_bytes_per_step": e2e["d2h"],
                           "ms_per_step": e2e["ms"], "api": "tc_rk4_step (host pointers, pinned)"}
        if world == 1 and not args.quick:
            line["adjoint"] = time_adjoint(device)
            line["batched"] = time_batch(device)
            line["rh4_l4_fp64"] = time_config1(device, check=not args.no_cpu)
            if args.config != "gaussian_l7":
                line["gaussian_l7"] = time_side_workload("gaussian_l7", device, args.no_cpu)
        if world == 1 and not args.no_cpu:
            threads = os.cpu_count() or 1
            # the CPU legs run on the oracle's own grid (bit for bit the library's inputs)
            wo = oracle_workload(args.config, check=w)
            frac = sample_frac(wo, 10.0, threads)
            cb = cpu_baseline(wo, frac=frac, threads=threads)
            line["cpu_baseline"] = {"value": cb["value"], "unit": "interactions/s", "cores": cb["cores"],
                                    "kind": "port", "sample": cb["sample"], "seconds": cb["seconds"],
                                    "build": cb["build"], "inputs": "oracle grid (oracle/icos_oracle.c)",
                                    "pinned": PORT_PINNED}
            line["error_vs_fp64_oracle"] = error_sample(wo, device, threads)
        print(json.dumps(line), flush=True)
    main["ctx"].close() if driver is None else driver.close()


# what ties the timed C port to the reference: its strict build equals, bit for bit, the
# reference's own Fortran statements run through the Fortran 90 subset translator (oracle/f90)
PORT_PINNED = ("strict build equal bit for bit to the reference's own Fortran source (grid, initial "
               "conditions, BVERK4 on 1-5 MPI ranks, StratosphereRK4, the sums) run through oracle/f90; "
               "the timed build agrees with the strict one to 1e-12")


def repo_libraries() -> list[str]:
    """Shared libraries of this repository mapped into the process (from /proc/self/maps)."""
    try:
        with open("/proc/self/maps") as f:
            paths = {ln.split()[-1] for ln in f if ln.rstrip().endswith(".so")}
    except OSError:
        return []
    return sorted(os.path.relpath(q, ROOT) for q in paths if q.startswith(str(ROOT)))


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    w = oracle_workload(args.config)  # the oracle's grid: no part of the product library is loaded
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_baseline(w, frac=1.0 / 1024, threads=threads)
    frac = sample_frac(w, 2.0, threads, lo=1.0 / 1024)
    vals, secs = [], []
    for _ in range(args.steps):
        cb = cpu_baseline(w, frac=frac, threads=threads)
        vals.append(cb["value"])
        secs.append(cb["seconds"])
    v = statistics.median(vals)
    line = {"impl": "reference", "metric": "Biot-Savart interactions/s (one RK4 step of the direct spherical sum)",
            "value": v, "unit": "interactions/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": w.interactions_per_step() / v * 1e3, "higher_is_better": True,
            "scaling": "strong" if world > 1 else "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: analytic vorticity on a generated icosahedral grid (seeded)",
            "config": workload_config(w, "fp64 (CPU)", "host cores"),
            "cpu_baseline": {"value": v, "unit": "interactions/s", "cores": threads, "kind": "port",
                             "sample": cb["sample"] + "; each step one such sample, rate extrapolated linearly",
                             "build": cb["build"], "pinned": PORT_PINNED},
            "e2e": {"value": v, "unit": "interactions/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference is Fortran+MPI (ifort -O2, mpif90); no Fortran compiler or MPI exists on "
                    "these machines, so the arm runs the C restatement of its loops (oracle/), compiled with "
                    "the floating-point freedoms and vectorization of ifort -O2, on all host threads with the "
                    "reference's LoadBalance row partition, on inputs from the oracle's restatement of the "
                    "reference's icosahedral grid generator (InitIcosTriGrid/DivideTriPanel)"}
    line["libraries_loaded"] = repo_libraries()
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="rh4_l8", choices=["rh4_l8", "gaussian_l7", "rh4_l4", "jet_l6"])
    ap.add_argument("--precision", default="fp32c", choices=["fp32c", "fp64"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline and error check")
    ap.add_argument("--quick", action="store_true", help="main measurement only")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
