"""Benchmark: multimode Rayleigh + Love dispersion roots/s on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one "step"): the batched crustal configuration -- 10,000 seeded random
models with 8-20 layers over a half-space (padded to 21 rows), 60 periods
geomspaced 0.5-50 s, 5 modes, Rayleigh and Love, group velocity on -- solved to
c_tol_rel 1e-10 (|dc|/c <= 1e-11, inside the 1e-9 parity bar).  Each rank solves
its own batch (weak scaling; ranks exchange nothing but the timing reduction).

Printed JSON (rank 0, one line):
  value      roots/s of the FP32-scan / FP64-refinement engine, device-resident
             inputs, CUDA events on the launching stream, L2 flushed between steps
  e2e        the same metric through the plugin's QeSolver.run (C ABI host path,
             host arrays, host<->device copies inside the timed region)
  fp64       the plain FP64 engine on the same protocol (the denominator of the
             FP32-scan speed-up)
  roofline   the scan kernel's algorithmic FP32 flop rate against the measured
             non-tensor FP32 FMA peak of this GPU
  cpu_baseline  the reference CPU engine (oracle/_ref, built from the reference
             sources) on a bounded sample of the same batch, all host cores
--impl reference times that reference CPU engine alone (rank 0 only).
"""
from __future__ import annotations

import argparse
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

METRIC = "roots/s at |dc/c|<=1e-9 (FP32-scan+FP64-refine engine; plain FP64 alongside)"
TOL = 1e-10
MODELS = 10_000
WORKLOAD = "crustal batch: 10000 models x 8-20 layers, 60 periods 0.5-50 s, 5 modes, Rayleigh+Love, group velocity"
# Algorithmic floating-point operations of one layer step of the secular
# recurrences, counted from modisp_b200/csrc/secular.cuh (adds and multiplies
# each 1, an FMA 2; the elementary functions counted separately: 2 rsqrt and
# 2 sin/cos-or-exp per Rayleigh step, 1 rsqrt and 1 sin/cos-or-exp per Love step).
FLOPS_PER_STEP = {0: 170, 1: 24}
# DRAM traffic of the FP32 Rayleigh scan, dram__bytes_read.sum + dram__bytes_write.sum
# from one ncu capture of a 2,000-model launch (120,000 traces: 30.1 MB + 93.0 MB),
# per trace; scaled to this workload's launch by its trace count.
SCAN32_DRAM_BYTES_PER_TRACE = (30.661888e6 + 95.3536e6) / 120_000


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=("ours", "reference"), default="ours")
    p.add_argument("--models", type=int, default=MODELS)
    p.add_argument("--cpu-sample", type=int, default=128, help="models in the CPU-baseline sample")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-jacobian", action="store_true")
    p.add_argument("--no-ragged", action="store_true")
    p.add_argument("--no-config3", action="store_true")
    p.add_argument("--no-reliability", action="store_true")
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    return rank, world, local


def workload(rank, models):
    from modisp_b200 import workloads
    batch = workloads.crustal_batch(models, seed=workloads.SEED + 2 + 1000 * rank)
    return batch, np.geomspace(0.5, 50., 60), 5


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    def __init__(self, index):
        self.index, self.proc, self.lines = index, None, []

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for name, flag in zip(names, parts[4:8]):
                if flag.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline(batch, periods, nmodes, sample):
    """The reference CPU engine (built from the reference sources) on a bounded sample."""
    import oracle
    ref = oracle.reference()
    if ref is None:
        return None
    sub = {k: v[:sample] for k, v in batch.items()}
    cores = len(os.sched_getaffinity(0))
    threads = min(256, cores)
    roots, elapsed = 0, 0.
    for wave in (0, 1):
        oracle.reference_solve(sub["thickness"][:4], sub["vp"][:4], sub["vs"][:4], sub["rho"][:4], periods, nmodes,
                               wave=wave, tol=TOL, threads=threads, group_velocity=True)  # warm-up
        t = time.perf_counter()
        out = oracle.reference_solve(sub["thickness"], sub["vp"], sub["vs"], sub["rho"], periods, nmodes,
                                     wave=wave, tol=TOL, threads=threads, group_velocity=True)
        elapsed += time.perf_counter() - t
        roots += int(np.isfinite(out["phase_velocity"]).sum())
    return {"value": roots / elapsed, "unit": "roots/s", "cores": threads, "kind": "reference", "seconds": elapsed,
            "sample": f"{sample} models of the same batch x 60 periods x 5 modes, Rayleigh+Love, group velocity, "
                      f"accuracy=high shape-adaptive, c_tol_rel={TOL:g}; {roots} roots in {elapsed:.2f} s"}


def run_reference(args, rank, world):
    if rank != 0:
        return
    batch, periods, nmodes = workload(0, args.models)
    sample = args.cpu_sample
    vals, times = [], []
    for step in range(args.warmup + args.steps):
        res = cpu_baseline(batch, periods, nmodes, sample)
        if res is None:
            print(json.dumps({"impl": "reference", "unavailable": "reference CPU engine not built (make -C oracle)"}))
            return
        if step >= args.warmup:
            vals.append(res["value"])
            times.append(res["seconds"])
    value = statistics.median(vals)
    line = {"metric": METRIC, "value": value, "unit": "roots/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * statistics.median(times), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)", "impl": "reference",
            "config": {"workload": WORKLOAD, "models_per_step": sample, "periods": 60, "nmodes": 5,
                       "c_tol_rel": TOL},
            "cpu_baseline": {"value": value, "unit": "roots/s", "cores": res["cores"], "kind": "reference",
                             "sample": res["sample"]},
            "e2e": {"value": value, "unit": "roots/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def jacobian_bench(torch, local, steps, warmup, flush):
    """Differentiation workload: forward solve, full phase/group Jacobians and the
    misfit gradient (vector-Jacobian product) of 4096 12-layer models, 40 periods
    1-40 s, 3 modes, Rayleigh, timed separately with CUDA events."""
    from modisp_b200 import _native, workloads
    batch, periods, nmodes = workloads.config4(4096)
    B, L = batch["thickness"].shape
    T = periods.size
    dev = torch.device("cuda", local)
    f64 = torch.float64
    x = {k: torch.tensor(batch[k], dtype=f64, device=dev) for k in ("thickness", "vp", "vs", "rho")}
    per = torch.tensor(periods, dtype=f64, device=dev)
    vel = torch.empty((B, nmodes, T), dtype=f64, device=dev)
    grp = torch.empty_like(vel)
    gfl = torch.empty((B, nmodes, T), dtype=torch.int32, device=dev)
    i32 = [torch.empty((B, T), dtype=torch.int32, device=dev) for _ in range(3)]
    jc = torch.empty((B, nmodes, T, 4, L), dtype=f64, device=dev)
    ju = torch.empty_like(jc)
    grad = torch.empty((4, B, L), dtype=f64, device=dev)
    w = torch.ones_like(vel)
    o = _native.default_options()
    o.single_precision = 1
    o.group_velocity = 1
    eng = _native.Engine(local, B, L, T, nmodes, o)
    stream = torch.cuda.current_stream().cuda_stream
    ptrs = [x[k].data_ptr() for k in ("thickness", "vp", "vs", "rho")]

    def forward():
        eng.run_device(*ptrs, B, per.data_ptr(), 0, TOL, 1., 0, vel.data_ptr(), i32[0].data_ptr(),
                       i32[1].data_ptr(), i32[2].data_ptr(), grp.data_ptr(), gfl.data_ptr(), stream=stream)

    def full():
        eng.jacobian_device(*ptrs, B, per.data_ptr(), 0, vel.data_ptr(), jc.data_ptr(), group=grp.data_ptr(),
                            jac_group=ju.data_ptr(), stream=stream)

    def vjp():
        eng.vjp_device(*ptrs, B, per.data_ptr(), 0, vel.data_ptr(), grad.data_ptr(), weight_phase=w.data_ptr(),
                       weight_group=w.data_ptr(), group=grp.data_ptr(), stream=stream)

    def timed(fn):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        total = 0.
        for _ in range(steps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            b.synchronize()
            total += a.elapsed_time(b)
        return total / steps

    ms_f = timed(forward)
    roots = int(torch.isfinite(vel).sum())
    ms_j = timed(full)
    ms_v = timed(vjp)
    nan_rows = int(torch.isnan(jc[..., 0, 0][torch.isfinite(vel)]).sum())
    eng.close()
    return {"workload": "4096 models x 12 layers + half-space, 40 periods 1-40 s, 3 modes, Rayleigh, "
                        "Jacobians of phase and group velocity w.r.t. h, Vp, Vs, rho of every row",
            "roots": roots, "forward_ms": ms_f, "jacobian_ms": ms_j, "vjp_ms": ms_v,
            "jacobian_roots_per_s": roots / ((ms_f + ms_j) * 1e-3),
            "gradient_roots_per_s": roots / ((ms_f + ms_v) * 1e-3),
            "jacobian_cost_ratio": ms_j / ms_f, "vjp_cost_ratio": ms_v / ms_f,
            "failed_roots": nan_rows, "unit": "roots/s"}


RAGGED_MODELS = 10_000


def config3_bench(torch, local, flush, sample=256, rank=0):
    """Mixed precision on the 100,000-model batch with 30 % low-velocity-layer models:
    FP32-scan throughput (one timed step, both waves), agreement of the FP32-scan and
    plain FP64 engines over the whole batch, and per-root error of the FP32-scan
    engine against the reference CPU engine on a sample of the batch."""
    from modisp_b200 import _native, workloads
    import oracle
    batch, periods, nmodes = workloads.config3()
    B, L = batch["thickness"].shape
    T = periods.size
    dev = torch.device("cuda", local)
    x = {k: torch.tensor(batch[k], device=dev) for k in ("thickness", "vp", "vs", "rho")}
    per = torch.tensor(periods, device=dev)
    out = {}
    ms = 0.
    for single in (1, 0):
        o = _native.default_options()
        o.single_precision = single
        o.group_velocity = 1
        eng = _native.Engine(local, B, L, T, nmodes, o)
        stream = torch.cuda.current_stream().cuda_stream
        for wave in (0, 1):
            vel = torch.empty((B, nmodes, T), dtype=torch.float64, device=dev)
            grp = torch.empty_like(vel)
            gfl = torch.empty((B, nmodes, T), dtype=torch.int32, device=dev)
            tr = [torch.empty((B, T), dtype=torch.int32, device=dev) for _ in range(3)]
            args = (x["thickness"].data_ptr(), x["vp"].data_ptr(), x["vs"].data_ptr(), x["rho"].data_ptr(), B,
                    per.data_ptr(), 0, TOL, 1., wave, vel.data_ptr(), tr[0].data_ptr(), tr[1].data_ptr(),
                    tr[2].data_ptr(), grp.data_ptr(), gfl.data_ptr())
            eng.run_device(*args, stream=stream)  # warm-up
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            eng.run_device(*args, stream=stream)
            b.record()
            b.synchronize()
            if single:
                ms += a.elapsed_time(b)
            out[single, wave] = (vel.cpu().numpy(), grp.cpu().numpy(), tr[2].cpu().numpy())
        eng.close()
    roots = sum(int(np.isfinite(out[1, w][0]).sum()) for w in (0, 1))
    agree = {"mask_mismatch_traces": 0, "count_mismatches": 0, "max_rel_diff_phase": 0., "max_rel_diff_group": 0.}
    for w in (0, 1):
        v32, g32, c32 = out[1, w]
        v64, g64, c64 = out[0, w]
        agree["mask_mismatch_traces"] += int(np.any(np.isfinite(v32) != np.isfinite(v64), axis=1).sum())
        agree["count_mismatches"] += int((c32 != c64).sum())
        m = np.isfinite(v32) & np.isfinite(v64)
        agree["max_rel_diff_phase"] = max(agree["max_rel_diff_phase"], float((np.abs(v32[m] - v64[m]) / v64[m]).max()))
        mg = np.isfinite(g32) & np.isfinite(g64)
        agree["max_rel_diff_group"] = max(agree["max_rel_diff_group"], float((np.abs(g32[mg] - g64[mg]) / g64[mg]).max()))
    vs_ref = None
    if rank == 0 and oracle.reference() is not None:
        threads = len(os.sched_getaffinity(0))
        idx = np.linspace(0, B - 1, sample).astype(int)
        vs_ref = {"sample_models": sample, "mask_mismatch_traces": 0, "count_mismatches": 0, "max_rel_err_phase": 0.}
        for w in (0, 1):
            ref = oracle.reference_solve(*(batch[k][idx] for k in ("thickness", "vp", "vs", "rho")), periods, nmodes,
                                         wave=w, tol=1e-12, threads=threads)
            v, rv = out[1, w][0][idx], ref["phase_velocity"]
            vs_ref["mask_mismatch_traces"] += int(np.any(np.isfinite(v) != np.isfinite(rv), axis=1).sum())
            vs_ref["count_mismatches"] += int((out[1, w][2][idx] != ref["root_count"]).sum())
            m = np.isfinite(v) & np.isfinite(rv)
            vs_ref["max_rel_err_phase"] = max(vs_ref["max_rel_err_phase"], float((np.abs(v[m] - rv[m]) / rv[m]).max()))
    return {"workload": "100,000 models as the crustal batch, 30 % with one low-velocity layer (Vs 20-40 % below "
                        "the layer above), 60 periods 0.5-50 s, 5 modes, Rayleigh + Love, FP32 scan / FP64 refinement",
            "value": roots / (ms * 1e-3), "unit": "roots/s", "ms_per_step": ms, "roots_per_step": roots,
            "fp32_vs_fp64_engine": agree, "fp32_vs_reference": vs_ref}


def hbm_peak_gbs():
    """Measured HBM copy bandwidth of this pool's B200s (MEASURED_PEAKS.json), else the fallback."""
    try:
        return float(json.loads((Path(__file__).resolve().parent / "MEASURED_PEAKS.json").read_text())["hbm_gbs"]), \
            "measured"
    except (OSError, ValueError, KeyError):
        return 6650., "fallback"


def reliability_bench(torch, local, steps, flush, rank=0, sample=300):
    """Cross-period mode-reliability checks of a solved crustal batch (10,000 models
    x 5 modes x 60 periods, Rayleigh, FP32-scan engine): the kernel on device buffers
    timed with CUDA events (L2 flushed before each step), the public
    check_mode_reliability on host arrays (copies included, wall clock), and the
    oracle port on a bounded sample of the same result, whose flags the kernel's
    must match bit for bit (the checks are per model, so a sample of models is a
    sample of the job)."""
    from modisp_b200 import _native, workloads
    from modisp_b200.reliability import check_mode_reliability, period_plan
    import oracle.reliability as orel
    batch, periods, nmodes = workloads.config2()
    B, L = batch["thickness"].shape
    T = periods.size
    o = _native.default_options()
    o.single_precision = 1
    eng = _native.Engine(local, B, L, T, nmodes, o)
    out = eng.run(batch["thickness"], batch["vp"], batch["vs"], batch["rho"], periods, None, TOL, 1., 0)
    eng.close()
    v = np.ascontiguousarray(out["velocity"], dtype=np.float64)
    tf = np.ascontiguousarray(out["flags"], dtype=np.uint32)
    cnt = np.ascontiguousarray(out["counts"], dtype=np.int64)
    dev = torch.device("cuda", local)
    v_d = torch.tensor(v, device=dev)
    tf_d = torch.tensor(tf.view(np.int32), device=dev)
    cnt_d = torch.tensor(cnt, device=dev)
    fl_d = torch.empty((B, nmodes, T), dtype=torch.int16, device=dev)
    as_d = torch.empty((B, nmodes, T), dtype=torch.uint8, device=dev)
    plan, order, _ = period_plan(periods)
    stream = torch.cuda.current_stream().cuda_stream

    plan_d = torch.tensor(plan.view(np.uint8), device=dev)
    order_d = torch.tensor(order, device=dev)

    def device_call():  # plan uploaded by the call (stream-ordered scratch)
        _native.mode_reliability_device(v_d.data_ptr(), tf_d.data_ptr(), cnt_d.data_ptr(), B, nmodes, T, plan, order,
                                        .005, .1, .05, fl_d.data_ptr(), as_d.data_ptr(), stream)

    def kernel_call():  # plan already on the device: the kernel alone
        _native.mode_reliability_planned(v_d.data_ptr(), tf_d.data_ptr(), cnt_d.data_ptr(), B, nmodes, T,
                                         plan_d.data_ptr(), order_d.data_ptr(), .005, .1, .05, fl_d.data_ptr(),
                                         as_d.data_ptr(), stream)

    def timed(call):
        for _ in range(3):
            call()
        total = 0.
        for _ in range(steps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            call()
            b.record()
            b.synchronize()
            total += a.elapsed_time(b)
        return total / steps

    ms_upload = timed(device_call)
    ms = timed(kernel_call)
    check_mode_reliability(v, periods, trace_flags=tf, root_count=cnt, device=local)  # warm-up
    t0 = time.perf_counter()
    for _ in range(steps):
        res = check_mode_reliability(v, periods, trace_flags=tf, root_count=cnt, device=local)
    wall = (time.perf_counter() - t0) / steps
    same_device = bool(np.array_equal(fl_d.cpu().numpy().view(np.uint16), res.flags))
    cells = B * nmodes * T
    algorithmic = cells * (8 + 2 + 1) + B * T * (4 + 8)  # roots in; flags, assessed out; trace flags, counts in
    peak, peak_kind = hbm_peak_gbs()
    line = {"workload": "check_mode_reliability of a solved 10,000-model crustal result (5 modes x 60 periods, "
                        "Rayleigh, FP32-scan engine), default thresholds",
            "cells_per_step": cells, "flagged_fraction": float((res.flags != 0).mean()),
            "value": cells / (ms * 1e-3), "unit": "cells/s", "ms_per_step": ms,
            "roofline": {"bound": "hbm", "kernel": "mode_reliability", "achieved": algorithmic / (ms * 1e-3) / 1e9,
                         "peak": peak, "unit": "GB/s", "frac": algorithmic / (ms * 1e-3) / 1e9 / peak,
                         "peak_kind": peak_kind, "algorithmic_bytes": algorithmic},
            "ms_per_step_with_plan_upload": ms_upload,
            "e2e": {"value": cells / wall, "unit": "cells/s", "ms_per_step": wall * 1e3,
                    "h2d_bytes_per_step": v.nbytes + tf.nbytes + cnt.nbytes + plan.nbytes + order.nbytes,
                    "d2h_bytes_per_step": cells * 3},
            "device_and_host_entry_agree": same_device}
    if rank == 0:
        idx = np.linspace(0, B - 1, sample).astype(int)
        t0 = time.perf_counter()
        want = orel.check(v[idx], periods, tf[idx], cnt[idx])
        cpu_s = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": sample * nmodes * T / cpu_s, "unit": "cells/s", "cores": 1, "kind": "port",
                                "sample": f"{sample} of the 10,000 models ({sample * nmodes * T} cells), the oracle's "
                                          f"numpy restatement vectorised as the reference's; {cpu_s:.2f} s"}
        line["matches_oracle_on_sample"] = bool(np.array_equal(res.flags[idx], want[0]) and
                                                np.array_equal(res.assessed[idx], want[1]))
    return line


def ragged_bench(torch, local, steps, warmup, flush, models=RAGGED_MODELS):
    """Large uneven batch: smooth-gradient models of 30-100 thin layers, each with its
    own 50-120 periods inside 0.2-100 s and 1-10 modes, Rayleigh + Love, FP32 scan /
    FP64 refinement, group velocity; one ragged (CSR) run per wave, both captured in
    one CUDA graph that each step replays.  A seeded sample of the 1,000,000-model
    workload (throughput does not depend on the batch size beyond filling the GPU)."""
    from modisp_b200 import _native, workloads
    batch, periods, modes = workloads.gradient_batch(models, seed=workloads.SEED + 50)
    B, L = batch["thickness"].shape
    off = np.zeros(B + 1, np.int32)
    off[1:] = np.cumsum([p.size for p in periods])
    flat = np.concatenate(periods)
    md = np.asarray(modes, np.int32)
    cells = md.astype(np.int64) * np.diff(off)
    outb = np.zeros(B, np.int64)
    outb[1:] = np.cumsum(cells)[:-1]
    ntr, ncell = int(off[-1]), int(cells.sum())
    dev = torch.device("cuda", local)
    x = {k: torch.tensor(batch[k], device=dev) for k in ("thickness", "vp", "vs", "rho")}
    meta = {k: torch.tensor(v, device=dev) for k, v in (("off", off), ("per", flat), ("md", md), ("outb", outb))}
    vel = [torch.empty(ncell, dtype=torch.float64, device=dev) for _ in range(2)]
    grp = [torch.empty_like(v) for v in vel]
    gfl = [torch.empty(ncell, dtype=torch.int32, device=dev) for _ in range(2)]
    tr = [[torch.empty(ntr, dtype=torch.int32, device=dev) for _ in range(3)] for _ in range(2)]
    o = _native.default_options()
    o.single_precision = 1
    o.group_velocity = 1
    eng = _native.Engine(local, B, L, int(np.diff(off).max()), int(md.max()), o)
    eng.graph_begin()
    for wave in (0, 1):
        eng.run_ragged_device(x["thickness"].data_ptr(), x["vp"].data_ptr(), x["vs"].data_ptr(), x["rho"].data_ptr(),
                              B, ntr, meta["off"].data_ptr(), meta["per"].data_ptr(), meta["md"].data_ptr(),
                              meta["outb"].data_ptr(), TOL, 1., wave, vel[wave].data_ptr(), tr[wave][0].data_ptr(),
                              tr[wave][1].data_ptr(), tr[wave][2].data_ptr(), grp[wave].data_ptr(),
                              gfl[wave].data_ptr())
    eng.graph_end()
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(warmup):
        eng.graph_launch(stream)
    torch.cuda.synchronize()
    total = 0.
    for _ in range(steps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        eng.graph_launch(stream)
        b.record()
        b.synchronize()
        total += a.elapsed_time(b)
    roots = sum(int(torch.isfinite(v).sum()) for v in vel)
    unconverged = sum(int((t[2] < 0).sum()) for t in tr)
    eng.close()
    return {"workload": f"{B} of the 1,000,000 smooth-gradient models (30-100 layers over 0-80 km), own 50-120 "
                        "periods in 0.2-100 s, 1-10 modes each; Rayleigh + Love; ragged CSR batch, one CUDA graph",
            "models": B, "traces_per_wave": ntr, "output_cells_per_wave": ncell, "roots_per_step": roots,
            "ms_per_step": total / steps, "value": roots * steps / (total * 1e-3), "unit": "roots/s",
            "unconverged_traces": unconverged, "launches_per_step": eng_launches_ragged()}


def eng_launches_ragged():
    # prep, init, tail values, scan, refine, repair select, repair scan, repair refine, assemble, group: per wave
    return 2 * 10


def device_run(torch, eng, tens, B, wave, stream):
    """Enqueue one engine run on device-resident tensors."""
    eng.run_device(tens["h"].data_ptr(), tens["vp"].data_ptr(), tens["vs"].data_ptr(), tens["rho"].data_ptr(), B,
                   tens["per"].data_ptr(), 0, TOL, 1., wave, tens["vel"][wave].data_ptr(),
                   tens["flags"][wave].data_ptr(), tens["levels"][wave].data_ptr(), tens["counts"][wave].data_ptr(),
                   tens["grp"][wave].data_ptr(), tens["gfl"][wave].data_ptr(), None, None,
                   tens["stats"][wave].data_ptr(), stream)


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    import torch
    from modisp_b200 import _native, plugin, sharding

    torch.cuda.set_device(local)
    # a dedicated stream: the engine's kernels and the timing events share it
    work_stream = torch.cuda.Stream()
    torch.cuda.set_stream(work_stream)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    batch, periods, nmodes = workload(rank, args.models)
    B, L = batch["thickness"].shape
    T = periods.size
    dev = torch.device("cuda", local)
    f64 = torch.float64
    tens = {k: torch.tensor(batch[k], dtype=f64, device=dev) for k in ("thickness", "vp", "vs", "rho")}
    tens = {"h": tens["thickness"], "vp": tens["vp"], "vs": tens["vs"], "rho": tens["rho"],
            "per": torch.tensor(periods, dtype=f64, device=dev),
            "vel": [torch.empty((B, nmodes, T), dtype=f64, device=dev) for _ in range(2)],
            "grp": [torch.empty((B, nmodes, T), dtype=f64, device=dev) for _ in range(2)],
            "gfl": [torch.empty((B, nmodes, T), dtype=torch.int32, device=dev) for _ in range(2)],
            "flags": [torch.empty((B, T), dtype=torch.int32, device=dev) for _ in range(2)],
            "levels": [torch.empty((B, T), dtype=torch.int32, device=dev) for _ in range(2)],
            "counts": [torch.empty((B, T), dtype=torch.int32, device=dev) for _ in range(2)],
            "stats": [torch.zeros(_native.STAT_COUNT, dtype=torch.int64, device=dev) for _ in range(2)]}
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # 256 MiB > 126 MB L2

    # launch shape of the scan, chosen by the autotuner on a 1,000-model sample
    from modisp_b200 import autotune
    sample = {k: v[:1000] for k, v in batch.items()}
    tuned = {}
    for single in (True, False):
        tuned[single] = autotune.autotune(sample, periods, nmodes, 0, single, device=local, use_cache=False)

    def engine(single):
        o = _native.default_options()
        o.single_precision = int(single)
        o.group_velocity = 1
        autotune.apply(o, tuned[single])
        return _native.Engine(local, B, L, T, nmodes, o)

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    def timed(eng, steps, warmup):
        stream = torch.cuda.current_stream().cuda_stream
        for _ in range(warmup):
            for wave in (0, 1):
                device_run(torch, eng, tens, B, wave, stream)
        barrier()
        total = 0.
        for _ in range(steps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for wave in (0, 1):
                device_run(torch, eng, tens, B, wave, stream)
            b.record()
            b.synchronize()
            total += a.elapsed_time(b)
        barrier()
        roots = sum(int(torch.isfinite(tens["vel"][w]).sum()) for w in (0, 1))
        return total, roots

    def reduce_max(x):
        return sharding.reduce_max(x, dev)

    def reduce_sum(x):
        return sharding.reduce_sum(x, dev)

    # ---- FP32-scan engine: the headline ----
    e32 = engine(True)
    with ClockSampler(local) as clocks:
        ms32, roots32 = timed(e32, args.steps, args.warmup)
    ms32 = reduce_max(ms32)
    roots_all = reduce_sum(roots32)
    value = roots_all * args.steps / (ms32 * 1e-3)
    # per-stage device times of one more run per wave (scan kernel = dominant)
    stream = torch.cuda.current_stream().cuda_stream
    stage = {}
    scan_flops = 0.
    for wave in (0, 1):
        flush.zero_()
        device_run(torch, e32, tens, B, wave, stream)
        st = e32.stage_times()
        stats = tens["stats"][wave].cpu().numpy()
        stage[wave] = st
        scan_flops += float(stats[3]) * FLOPS_PER_STEP[wave]  # FP32 layer steps (scan kernel)
    scan_ms = sum(stage[w]["scan"] for w in (0, 1))
    launches = e32.kernel_launches() * 2 * args.steps
    e32_stats = {w: tens["stats"][w].cpu().numpy().tolist() for w in (0, 1)}

    # ---- plain FP64 engine ----
    e64 = engine(False)
    ms64, roots64 = timed(e64, max(2, args.steps // 2), 1)
    ms64 = reduce_max(ms64)
    value64 = reduce_sum(roots64) * max(2, args.steps // 2) / (ms64 * 1e-3)
    e64.close()

    # ---- end to end through the plugin (host arrays) ----
    h2d = d2h = 0
    e2e_value = None
    if True:
        solver = plugin.QeSolver(B, L, T, nmodes, 0, 0., .005, True, .001, 0, 1, 1, True, True, .001, False, 4,
                                 device=local)
        bounds = np.zeros((B, 2))
        bounds[:, 1] = np.inf
        host = [np.ascontiguousarray(batch[k]) for k in ("thickness", "vp", "vs", "rho")]
        for _ in range(max(1, args.warmup - 1)):
            for wave in (0, 1):
                solver.run(*host, periods, bounds, TOL, 1., wave)
        barrier()
        t0 = time.perf_counter()
        outs = {}
        for _ in range(args.steps):
            for wave in (0, 1):
                outs[wave] = solver.run(*host, periods, bounds, TOL, 1., wave)
        barrier()
        wall = reduce_max(time.perf_counter() - t0)
        # every step returns the same roots: counted once, outside the timed region
        roots_e2e = args.steps * sum(int(np.isfinite(outs[w][0]).sum()) for w in (0, 1))
        e2e_value = reduce_sum(roots_e2e) / wall
        per_wave_in = sum(a.nbytes for a in host) + periods.nbytes + bounds.nbytes
        per_wave_out = B * nmodes * T * (8 + 8 + 4) + B * T * 4 * 3 + B * 16 + 16 * 8
        h2d, d2h = 2 * per_wave_in, 2 * per_wave_out
        solver.close()

    jac = jacobian_bench(torch, local, max(2, args.steps // 2), 2, flush) if not args.no_jacobian else None
    ragged = ragged_bench(torch, local, max(2, args.steps // 2), 2, flush) if not args.no_ragged else None
    config3 = config3_bench(torch, local, flush, rank=rank) if not args.no_config3 else None
    reliability = (reliability_bench(torch, local, max(3, args.steps), flush, rank=rank)
                   if not args.no_reliability else None)

    peak32 = _native.measure_peak(local, fp64=False)
    peak64 = _native.measure_peak(local, fp64=True)
    achieved = scan_flops / (scan_ms * 1e-3)
    cpu = None
    if rank == 0 and not args.no_cpu:
        cpu = cpu_baseline(batch, periods, nmodes, args.cpu_sample)
    e32.close()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "roots/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms32 / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (seeded crustal models)",
            "config": {"workload": WORKLOAD, "models_per_gpu": B, "layers_padded": L, "periods": T, "nmodes": nmodes,
                       "waves": ["rayleigh", "love"], "c_tol_rel": TOL, "l2": "flushed between steps (256 MiB write)",
                       "parallelism": f"model-sharded x{world}",
                       "scan_launch_shape": {"fp32": list(tuned[True]), "fp64": list(tuned[False]),
                                             "chosen_by": "autotuner (warps per CTA, CTAs per SM)"}},
            "fp64": {"value": value64, "unit": "roots/s", "ms_per_step": ms64 / max(2, args.steps // 2),
                     "fp32_scan_speedup": value / value64},
            "e2e": {"value": e2e_value, "unit": "roots/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "roofline": {"bound": "fp32-cuda-core", "kernel": "scan<float>", "achieved": achieved / 1e12,
                         "peak": peak32 / 1e12, "unit": "TFLOP/s", "frac": achieved / peak32,
                         "traffic": SCAN32_DRAM_BYTES_PER_TRACE * B * T,
                         "traffic_note": "bytes per Rayleigh FP32 scan launch, from an ncu capture of 2,000 models "
                                         "scaled by traces; the algorithmic input is the model tables (~1.5 KB per "
                                         "model): the kernel is compute-bound, DRAM at 0.2 % of peak",
                         "peak_kind": "measured FMA throughput (md200_measure_peak), not MEASURED_PEAKS.json",
                         "fp64_peak": peak64 / 1e12, "scan_ms_per_step": scan_ms,
                         "stage_ms": {("rayleigh" if w == 0 else "love"): stage[w] for w in (0, 1)}},
            "cpu_baseline": cpu,
            "gpu_launches": launches,
            "clocks": clocks.summary(),
            "engine_stats": {"rayleigh": e32_stats[0], "love": e32_stats[1]},
            "jacobian": jac,
            "ragged": ragged,
            "config3": config3,
            "reliability": reliability,
        }
        print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
