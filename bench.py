"""Benchmark: multimode Rayleigh + Love dispersion roots/s on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one "step"): the mixed-precision configuration -- 100,000 seeded random
models with 8-20 layers over a half-space (padded to 21 rows), 30 % of them with
one low-velocity layer (Vs 20-40 % below the layer above), 60 periods geomspaced
0.5-50 s, 5 modes, Rayleigh and Love, group velocity on -- solved to c_tol_rel
1e-10 (|dc|/c <= 1e-11, inside the 1e-9 parity bar).  Each rank solves its own
batch (weak scaling; ranks exchange nothing but the timing reduction).

Printed JSON (rank 0, one line):
  value      roots/s of the FP32-scan / FP64-refinement engine, device-resident
             inputs, CUDA events on the launching stream, L2 flushed between steps
  fp64       the plain FP64 engine on the same protocol (the denominator of the
             FP32-scan speed-up)
  e2e        the same metric through the plugin's QeSolver.run (C ABI host path,
             host arrays, host<->device copies inside the timed region)
  roofline   the dominant kernel's (the split scan's FP32 Rayleigh evaluation
             kernel) algorithmic FP32 flop rate against the measured non-tensor
             FP32 FMA peak of this GPU; the whole scan stage's rate alongside
  cpu_baseline, cpu_baseline_auto
             the reference CPU engine (oracle/_ref, built from the reference
             sources) through the reference's own Solver on a bounded sample of
             the same batch, all host cores, at accuracy="high" (c_tol_rel 1e-10)
             and at its default accuracy="auto"
  reference_cuda
             the reference's own CUDA plugin compiled for sm_100a (oracle/_ref/cuda)
             on a sample of the same batch on this GPU: a same-GPU comparator
  config2, jacobian, ragged, reliability, parity
             side workloads: the 10,000-model crustal batch, Jacobians (config 4),
             the large uneven batch (config 5 sample, with and without anchor
             continuation), the mode-reliability checks, and the agreement of both
             engines with each other and with the reference
--impl reference times the reference CPU engine alone (rank 0 only).
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
MODELS = 100_000
WORKLOAD = ("mixed-precision batch: 100000 models x 8-20 layers, 30 % with one low-velocity layer, "
            "60 periods 0.5-50 s, 5 modes, Rayleigh+Love, group velocity")
# Algorithmic floating-point operations of one layer step of the secular
# recurrences, counted from modisp_b200/csrc/secular.cuh (adds and multiplies
# each 1, an FMA 2; the elementary functions counted separately: 2 rsqrt and
# 2 sin/cos-or-exp per Rayleigh step, 1 rsqrt and 1 sin/cos-or-exp per Love step).
FLOPS_PER_STEP = {0: 170, 1: 24}
# DRAM traffic of the split scan's Rayleigh evaluation kernel (split_eval32_pair) per
# FP32 layer step it evaluates: dram__bytes_read.sum + dram__bytes_write.sum over
# the 9 launches of one run (1,090.4 MB + 715.8 MB), from an ncu capture of 2,000
# mixed-precision models, divided by that run's evaluated layer steps
# (MD200_STAT_SPLIT_EVAL_STEPS, 437,558,855).
EVAL_DRAM_BYTES_PER_STEP = (1090352896 + 715775488) / 437558855


def split_rounds(n_traces):
    """Launches of the split scan's evaluation kernel in one run (the engine's
    split_rounds: an active set of up to 2^20 traces, 3 rounds per set + 6)."""
    cap = min(n_traces, 1 << 20)
    return min(64, 3 * (-(-n_traces // cap)) + 6)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=("ours", "reference"), default="ours")
    p.add_argument("--models", type=int, default=MODELS)
    p.add_argument("--cpu-sample", type=int, default=1024, help="models in the CPU-baseline sample")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-side", action="store_true", help="skip every side workload")
    p.add_argument("--no-jacobian", action="store_true")
    p.add_argument("--no-ragged", action="store_true")
    p.add_argument("--no-config2", action="store_true")
    p.add_argument("--no-reliability", action="store_true")
    p.add_argument("--no-reference-cuda", action="store_true")
    p.add_argument("--no-uniform", action="store_true")
    p.add_argument("--no-autotune", action="store_true",
                   help="the engine's default launch shape and scan form (4 warps per CTA, CTAs per SM "
                        "from registers, automatic scan form) instead of tuning them on a sample; for runs "
                        "under a profiler, whose serialised launches mislead the tuner")
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    return rank, world, local


def workload(rank, models):
    """Rank 0 solves exactly the seeded mixed-precision batch; other ranks their own seeds."""
    from modisp_b200 import workloads
    batch = workloads.crustal_batch(models, seed=workloads.SEED + 3 + 1000 * rank, lvz_fraction=0.3)
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


# ---------------------------------------------------------------------------
# the reference CPU engine (oracle/_ref) on a bounded sample
# ---------------------------------------------------------------------------
def cpu_solve(sub, periods, nmodes, wave, accuracy, threads):
    """One wave of the reference CPU engine, through the reference's own Solver when
    the oracle recipe staged it (its stock path, continuity screen and review
    included), else through its CpuSolver directly."""
    import oracle
    wrapper = oracle.reference_wrapper()
    if wrapper is not None:
        opts = dict(backend="cpu", threads=threads, group_velocity=True)
        if accuracy == "high":
            opts.update(accuracy="high", c_tol_rel=TOL)
        r = wrapper.dispersion_batch(sub["thickness"], sub["vp"], sub["vs"], sub["rho"], periods, nmodes,
                                     "love" if wave else "rayleigh", **opts)
        return r.phase_velocity
    if accuracy != "high":
        return None
    out = oracle.reference_solve(sub["thickness"], sub["vp"], sub["vs"], sub["rho"], periods, nmodes, wave=wave,
                                 tol=TOL, threads=threads, group_velocity=True)
    return out["phase_velocity"]


def cpu_baseline(batch, periods, nmodes, sample, accuracy="high"):
    """The reference CPU engine on the first `sample` models of the batch (both
    waves), one warm-up call per wave, all host cores."""
    import oracle
    if oracle.reference() is None:
        return None
    sub = {k: np.ascontiguousarray(v[:sample]) for k, v in batch.items()}
    threads = min(256, len(os.sched_getaffinity(0)))
    roots, elapsed = 0, 0.
    for wave in (0, 1):
        small = {k: v[:4] for k, v in sub.items()}
        if cpu_solve(small, periods, nmodes, wave, accuracy, threads) is None:  # warm-up
            return None
        t = time.perf_counter()
        v = cpu_solve(sub, periods, nmodes, wave, accuracy, threads)
        elapsed += time.perf_counter() - t
        roots += int(np.isfinite(v).sum())
    path = "the reference's Solver(backend='cpu')" if oracle.reference_wrapper() is not None else "its CpuSolver"
    setting = (f"accuracy='high', c_tol_rel={TOL:g}" if accuracy == "high"
               else "default accuracy='auto' (c_tol_rel 1e-5, continuity screen and review on)")
    return {"value": roots / elapsed, "unit": "roots/s", "cores": threads, "kind": "reference", "seconds": elapsed,
            "accuracy": accuracy,
            "sample": f"{sample} of the {batch['thickness'].shape[0]} models x 60 periods x 5 modes, Rayleigh+Love, "
                      f"group velocity, {setting}, via {path}; {roots} roots in {elapsed:.2f} s"}


def run_reference(args, rank, world):
    if rank != 0:
        return
    batch, periods, nmodes = workload(0, args.models)
    sample = args.cpu_sample
    vals, times = [], []
    res = None
    for step in range(args.warmup + args.steps):
        res = cpu_baseline(batch, periods, nmodes, sample)
        if res is None:
            print(json.dumps({"impl": "reference", "unavailable": "reference CPU engine not built (make -C oracle)"}))
            return
        if step >= args.warmup:
            vals.append(res["value"])
            times.append(res["seconds"])
    value = statistics.median(vals)
    auto = cpu_baseline(batch, periods, nmodes, sample, accuracy="auto")
    line = {"metric": METRIC, "value": value, "unit": "roots/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * statistics.median(times), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)", "impl": "reference",
            "config": {"workload": WORKLOAD, "models_per_step": sample, "periods": 60, "nmodes": 5,
                       "c_tol_rel": TOL, "same_config_note": f"each step solves {sample} of the "
                       f"{args.models} models (a bounded sample; roots/s is a per-root rate)"},
            "cpu_baseline": {"value": value, "unit": "roots/s", "cores": res["cores"], "kind": "reference",
                             "sample": res["sample"]},
            "cpu_baseline_auto": auto,
            "e2e": {"value": value, "unit": "roots/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ---------------------------------------------------------------------------
# the reference's CUDA plugin (sm_100a build) on this GPU
# ---------------------------------------------------------------------------
def reference_cuda_bench(batch, periods, nmodes, local, sample=10_000, ours=None):
    """The reference's own QeSolver (its CUDA plugin compiled for sm_100a from its
    sources) on the first `sample` models, both waves, FP64 and FP32 precision at
    accuracy='high' (shape-adaptive search), host arrays in and out like its
    wrapper's call; one warm-up and two timed calls per wave.  Masks compared with
    this engine's on the same models."""
    import oracle
    mod = oracle.reference_cuda()
    if mod is None:
        return {"unavailable": "reference CUDA plugin not built (make -C oracle ref-cuda REFERENCE=...)"}
    mod.set_device(local)
    sub = {k: np.ascontiguousarray(v[:sample]) for k, v in batch.items()}
    B, L = sub["thickness"].shape
    T = periods.size
    out = {}
    for single in (False, True):
        s = mod.QeSolver(B, L, T, nmodes, 0, 0., .005, True, .001, 0, 1, 1, single, True, .001, False, 4)
        total, roots, masks = 0., 0, {}
        try:
            for wave in (0, 1):
                bounds = oracle.reference().bounds(sub["thickness"], sub["vp"], sub["vs"], sub["rho"], wave, None,
                                                   None)
                args = (sub["thickness"], sub["vp"], sub["vs"], sub["rho"], periods, bounds, TOL, 1., wave, True)
                s.run(*args)
                for _ in range(2):
                    t = time.perf_counter()
                    r = s.run(*args)
                    total += time.perf_counter() - t
                roots += 2 * int(np.isfinite(r[0]).sum())
                masks[wave] = np.isfinite(r[0])
        finally:
            s.close()
        key = "fp32" if single else "fp64"
        out[key] = {"value": roots / total, "unit": "roots/s", "seconds": total}
        if ours is not None:
            out[key]["mask_mismatch_traces_vs_this_engine"] = int(sum(
                np.any(masks[w] != np.isfinite(ours[w][:sample]), axis=1).sum() for w in (0, 1)))
    out["sample"] = (f"{sample} models of the batch, accuracy='high' shape-adaptive, c_tol_rel={TOL:g}, group "
                     f"velocity, QeSolver.run on host arrays (the wrapper's call), 2 timed calls per wave")
    return out


def uniform_bench(local, models=10_000, nc=512, cmin=0.2, calls=2):
    """The legacy uniform-grid path (search_strategy="uniform") on the 10,000-model
    crustal batch, Rayleigh, 60 periods, 5 modes, nc 512 over [0.2, the largest
    half-space vs]: this engine's CoarseScan/Refine and, beside it, the reference's
    own CUDA stages (compiled for sm_100a) through the same calls as the legacy
    solver makes them (python/modisp/_legacy.py:300-340: upload, scan, refine,
    download of roots and flags); one warm-up and `calls` timed calls each."""
    import oracle
    from modisp_b200 import plugin, workloads
    batch, periods, nmodes = workloads.config2(models)
    h, vp, vs, rho = (np.ascontiguousarray(batch[k]) for k in ("thickness", "vp", "vs", "rho"))
    B, L = h.shape
    cmax = float(vs[:, -1].max())

    def arm(mod):
        scan, refine = mod.CoarseScan(B, L), mod.Refine(B, L)
        for stage in (scan, refine):
            stage.upload_periods(periods)
        scan.allocate(nc)
        refine.allocate(nc, nmodes)

        def call():
            for stage in (scan, refine):
                stage.upload_models(h, vp, vs, rho)
            scan.run(cmin, cmax, 256)
            refine.run(scan, cmin, cmax, 1e-6, 1., nmodes, 256)
            return refine.download(), refine.flags()

        call()
        t = time.perf_counter()
        for _ in range(calls):
            v, f = call()
        return (time.perf_counter() - t) / calls, v, f

    out = {"workload": f"{B} crustal models (8-20 layers), Rayleigh, 60 periods 0.5-50 s, {nmodes} modes, nc {nc}, "
                       f"cmin {cmin}, cmax {cmax:.4g}, c_tol_rel 1e-6; host arrays in and out, {calls} timed calls",
           "unit": "roots/s"}
    sec, v, f = arm(plugin)
    out["ours"] = {"value": int(np.isfinite(v).sum()) / sec, "seconds_per_call": sec}
    ref = oracle.reference_cuda()
    if ref is None:
        out["reference"] = {"unavailable": "reference CUDA plugin not built (make -C oracle ref-cuda REFERENCE=...)"}
        return out
    ref.set_device(local)
    rsec, rv, rf = arm(ref)
    out["reference"] = {"value": int(np.isfinite(rv).sum()) / rsec, "seconds_per_call": rsec}
    out["speedup"] = rsec / sec
    both = np.isfinite(v) & np.isfinite(rv)
    diff = np.zeros(v.shape, bool)
    diff[both] = v[both] != rv[both]
    differ = np.any(diff | (np.isfinite(v) != np.isfinite(rv)), axis=1) | (f != rf)  # [B, T] traces
    # below max(vs) / 16 the reference's single-precision recurrence loses signs; its
    # rejected brackets show as trace flags (1 unresolved, 2 relocated)
    out["agreement"] = {"traces": int(differ.size), "roots": int(np.isfinite(rv).sum()),
                        "mask_mismatch_traces": int(np.any(np.isfinite(v) != np.isfinite(rv), axis=1).sum()),
                        "differing_traces": int(differ.sum()),
                        "differing_traces_the_reference_flags": int((differ & (rf != 0)).sum()),
                        "differing_traces_with_a_root_below_max_vs_over_16": int(
                            (differ & np.any(np.fmin(v, rv) < vs.max(axis=1)[:, None, None] / 16., axis=1)).sum()),
                        "identical_roots": int((both & ~diff).sum()),
                        "max_abs_root_difference": float(np.abs(v[both] - rv[both]).max(initial=0.))}
    return out


# ---------------------------------------------------------------------------
# side workloads
# ---------------------------------------------------------------------------
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


def config2_bench(torch, local, steps, warmup, flush):
    """The 10,000-model crustal batch (no low-velocity layers), both engines, the
    headline's device-resident protocol."""
    from modisp_b200 import _native, workloads
    batch, periods, nmodes = workloads.config2()
    B, L = batch["thickness"].shape
    T = periods.size
    tens = device_tensors(torch, batch, periods, nmodes, local)
    out = {}
    for single in (True, False):
        o = _native.default_options()
        o.single_precision, o.group_velocity = int(single), 1
        eng = _native.Engine(local, B, L, T, nmodes, o)
        ms, roots, _ = timed_runs(torch, eng, tens, B, steps, warmup, flush)
        eng.close()
        out["fp32" if single else "fp64"] = {"value": roots * steps / (ms * 1e-3), "ms_per_step": ms / steps}
    out["fp32_scan_speedup"] = out["fp32"]["value"] / out["fp64"]["value"]
    out["workload"] = "10,000 crustal models x 8-20 layers (no low-velocity layers), 60 periods 0.5-50 s, 5 modes"
    out["unit"] = "roots/s"
    return out


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


def ragged_bench(torch, local, steps, warmup, flush, models=RAGGED_MODELS, continuation=False):
    """Large uneven batch: smooth-gradient models of 30-100 thin layers, each with its
    own 50-120 periods inside 0.2-100 s and 1-10 modes, Rayleigh + Love, FP32 scan /
    FP64 refinement, group velocity; one ragged (CSR) run per wave, both captured in
    one CUDA graph that each step replays.  A seeded sample of the 1,000,000-model
    workload (throughput does not depend on the batch size beyond filling the GPU).
    With `continuation`, each model's periods run with anchor continuation."""
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
    o.continuation = int(continuation)
    eng = _native.Engine(local, B, L, int(np.diff(off).max()), int(md.max()), o)
    launches = 0
    eng.graph_begin()
    for wave in (0, 1):
        eng.run_ragged_device(x["thickness"].data_ptr(), x["vp"].data_ptr(), x["vs"].data_ptr(), x["rho"].data_ptr(),
                              B, ntr, meta["off"].data_ptr(), meta["per"].data_ptr(), meta["md"].data_ptr(),
                              meta["outb"].data_ptr(), TOL, 1., wave, vel[wave].data_ptr(), tr[wave][0].data_ptr(),
                              tr[wave][1].data_ptr(), tr[wave][2].data_ptr(), grp[wave].data_ptr(),
                              gfl[wave].data_ptr())
        launches += eng.kernel_launches()  # counted as the run enqueued them
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
            "unconverged_traces": unconverged, "launches_per_step": launches}


# ---------------------------------------------------------------------------
# the headline
# ---------------------------------------------------------------------------
def device_tensors(torch, batch, periods, nmodes, local):
    from modisp_b200 import _native
    B = batch["thickness"].shape[0]
    T = periods.size
    dev = torch.device("cuda", local)
    f64 = torch.float64
    t = {k: torch.tensor(batch[k], dtype=f64, device=dev) for k in ("thickness", "vp", "vs", "rho")}
    return {"h": t["thickness"], "vp": t["vp"], "vs": t["vs"], "rho": t["rho"],
            "per": torch.tensor(periods, dtype=f64, device=dev),
            "vel": [torch.empty((B, nmodes, T), dtype=f64, device=dev) for _ in range(2)],
            "grp": [torch.empty((B, nmodes, T), dtype=f64, device=dev) for _ in range(2)],
            "gfl": [torch.empty((B, nmodes, T), dtype=torch.int32, device=dev) for _ in range(2)],
            "flags": [torch.empty((B, T), dtype=torch.int32, device=dev) for _ in range(2)],
            "levels": [torch.empty((B, T), dtype=torch.int32, device=dev) for _ in range(2)],
            "counts": [torch.empty((B, T), dtype=torch.int32, device=dev) for _ in range(2)],
            "stats": [torch.zeros(_native.STAT_COUNT, dtype=torch.int64, device=dev) for _ in range(2)]}


def device_run(eng, tens, B, wave, stream):
    """Enqueue one engine run on device-resident tensors."""
    eng.run_device(tens["h"].data_ptr(), tens["vp"].data_ptr(), tens["vs"].data_ptr(), tens["rho"].data_ptr(), B,
                   tens["per"].data_ptr(), 0, TOL, 1., wave, tens["vel"][wave].data_ptr(),
                   tens["flags"][wave].data_ptr(), tens["levels"][wave].data_ptr(), tens["counts"][wave].data_ptr(),
                   tens["grp"][wave].data_ptr(), tens["gfl"][wave].data_ptr(), None, None,
                   tens["stats"][wave].data_ptr(), stream)


def timed_runs(torch, eng, tens, B, steps, warmup, flush, barrier=None):
    """W warm-up steps, then K timed steps (both waves each), L2 flushed before each
    step, CUDA events on the launching stream.  Returns (total ms, roots of one
    step, kernels launched per step)."""
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(warmup):
        for wave in (0, 1):
            device_run(eng, tens, B, wave, stream)
    (barrier or torch.cuda.synchronize)()
    total, launches = 0., 0
    for _ in range(steps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        launches = 0
        for wave in (0, 1):
            device_run(eng, tens, B, wave, stream)
            launches += eng.kernel_launches()
        b.record()
        b.synchronize()
        total += a.elapsed_time(b)
    (barrier or torch.cuda.synchronize)()
    roots = sum(int(torch.isfinite(tens["vel"][w]).sum()) for w in (0, 1))
    return total, roots, launches


def parity_summary(out32, out64, batch, periods, nmodes, rank, sample=256):
    """Agreement of the two engines on the whole headline batch, and of the FP32-scan
    engine with the reference CPU engine on a spread sample of it."""
    import oracle
    agree = {"mask_mismatch_traces": 0, "count_mismatches": 0, "max_rel_diff_phase": 0., "max_rel_diff_group": 0.}
    for w in (0, 1):
        v32, g32, c32 = out32[w]
        v64, g64, c64 = out64[w]
        agree["mask_mismatch_traces"] += int(np.any(np.isfinite(v32) != np.isfinite(v64), axis=1).sum())
        agree["count_mismatches"] += int((c32 != c64).sum())
        m = np.isfinite(v32) & np.isfinite(v64)
        agree["max_rel_diff_phase"] = max(agree["max_rel_diff_phase"], float((np.abs(v32[m] - v64[m]) / v64[m]).max()))
        mg = np.isfinite(g32) & np.isfinite(g64)
        agree["max_rel_diff_group"] = max(agree["max_rel_diff_group"],
                                          float((np.abs(g32[mg] - g64[mg]) / g64[mg]).max()))
    line = {"fp32_vs_fp64_engine": agree}
    if rank == 0 and oracle.reference() is not None:
        threads = len(os.sched_getaffinity(0))
        B = batch["thickness"].shape[0]
        idx = np.linspace(0, B - 1, sample).astype(int)
        vs_ref = {"sample_models": sample, "mask_mismatch_traces": 0, "count_mismatches": 0, "max_rel_err_phase": 0.}
        for w in (0, 1):
            ref = oracle.reference_solve(*(batch[k][idx] for k in ("thickness", "vp", "vs", "rho")), periods, nmodes,
                                         wave=w, tol=1e-12, threads=threads)
            v, rv = out32[w][0][idx], ref["phase_velocity"]
            vs_ref["mask_mismatch_traces"] += int(np.any(np.isfinite(v) != np.isfinite(rv), axis=1).sum())
            vs_ref["count_mismatches"] += int((out32[w][2][idx] != ref["root_count"]).sum())
            m = np.isfinite(v) & np.isfinite(rv)
            vs_ref["max_rel_err_phase"] = max(vs_ref["max_rel_err_phase"],
                                              float((np.abs(v[m] - rv[m]) / rv[m]).max()))
        line["fp32_vs_reference"] = vs_ref
    return line


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
    tens = device_tensors(torch, batch, periods, nmodes, local)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=torch.device("cuda", local))  # > L2

    # launch shape and FP32 scan form, chosen by the autotuner on a 1,000-model sample
    from modisp_b200 import autotune
    sample = {k: v[:1000] for k, v in batch.items()}
    tuned = {single: ((4, 0, 0) if args.no_autotune else
                      autotune.autotune(sample, periods, nmodes, None, single, device=local, use_cache=False))
             for single in (True, False)}

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

    def reduce_max(x):
        return sharding.reduce_max(x, torch.device("cuda", local))

    def reduce_sum(x):
        return sharding.reduce_sum(x, torch.device("cuda", local))

    def host_outputs():
        return {w: (tens["vel"][w].cpu().numpy(), tens["grp"][w].cpu().numpy(), tens["counts"][w].cpu().numpy())
                for w in (0, 1)}

    # ---- FP32-scan engine: the headline ----
    e32 = engine(True)
    with ClockSampler(local) as clocks:
        ms32, roots32, launches = timed_runs(torch, e32, tens, B, args.steps, args.warmup, flush, barrier)
    ms32 = reduce_max(ms32)
    value = reduce_sum(roots32) * args.steps / (ms32 * 1e-3)
    out32 = host_outputs()
    # per-stage device times of one more run per wave (the scan kernel dominates)
    stream = torch.cuda.current_stream().cuda_stream
    stage, scan_flops = {}, 0.
    for wave in (0, 1):
        flush.zero_()
        device_run(e32, tens, B, wave, stream)
        stage[wave] = e32.stage_times()
        stats = tens["stats"][wave].cpu().numpy()
        scan_flops += float(stats[3]) * FLOPS_PER_STEP[wave]  # FP32 layer steps the scans consumed
        if wave == 0:  # the dominant kernel: the split scan's FP32 evaluations (Rayleigh)
            eval_flops = float(stats[19]) * FLOPS_PER_STEP[0]
            eval_steps = float(stats[19])
    scan_ms = sum(stage[w]["scan"] for w in (0, 1))
    eval_ms = stage[0]["scan_eval"]
    eval_launches = split_rounds(B * T)
    e32_stats = {w: tens["stats"][w].cpu().numpy().tolist() for w in (0, 1)}
    e32.close()

    # ---- plain FP64 engine, same protocol ----
    e64 = engine(False)
    ms64, roots64, _ = timed_runs(torch, e64, tens, B, args.steps, args.warmup, flush, barrier)
    ms64 = reduce_max(ms64)
    value64 = reduce_sum(roots64) * args.steps / (ms64 * 1e-3)
    out64 = host_outputs()
    stage64 = {}
    for wave in (0, 1):
        flush.zero_()
        device_run(e64, tens, B, wave, stream)
        stage64[wave] = e64.stage_times()
    e64.close()
    del tens

    # ---- end to end through the plugin (host arrays) ----
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
    # device-to-host copies of one run: phase and group velocity (float64; the plugin
    # narrows phase to float32 on the host), group flags, trace flags, levels,
    # counts, windows and counters
    cells, traces = B * nmodes * T, B * T
    per_wave_out = cells * (8 + 8 + 4) + traces * 4 * 3 + B * 16 + _native.STAT_COUNT * 8
    solver.close()

    side = not args.no_side
    parity = parity_summary(out32, out64, batch, periods, nmodes, rank)
    config2 = (config2_bench(torch, local, max(2, args.steps // 2), 2, flush)
               if side and not args.no_config2 else None)
    jac = (jacobian_bench(torch, local, max(2, args.steps // 2), 2, flush)
           if side and not args.no_jacobian else None)
    ragged = None
    if side and not args.no_ragged:
        ragged = ragged_bench(torch, local, max(2, args.steps // 2), 2, flush)
        ragged["continuation"] = ragged_bench(torch, local, max(2, args.steps // 2), 2, flush, continuation=True)
    reliability = (reliability_bench(torch, local, max(3, args.steps), flush, rank=rank)
                   if side and not args.no_reliability else None)
    ref_cuda = (reference_cuda_bench(batch, periods, nmodes, local, ours={w: out64[w][0] for w in (0, 1)})
                if side and rank == 0 and not args.no_reference_cuda else None)
    uniform = uniform_bench(local) if side and rank == 0 and not args.no_uniform else None

    peak32 = _native.measure_peak(local, fp64=False)
    peak64 = _native.measure_peak(local, fp64=True)
    achieved = eval_flops / (eval_ms * 1e-3) if eval_ms > 0 else 0.
    scan_achieved = scan_flops / (scan_ms * 1e-3)
    cpu = cpu_auto = None
    if rank == 0 and not args.no_cpu:
        cpu = cpu_baseline(batch, periods, nmodes, args.cpu_sample)
        cpu_auto = cpu_baseline(batch, periods, nmodes, args.cpu_sample, accuracy="auto")
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "roots/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms32 / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic (seeded crustal models, 30 % with a low-velocity layer)",
            "config": {"workload": WORKLOAD, "models_per_gpu": B, "layers_padded": L, "periods": T, "nmodes": nmodes,
                       "waves": ["rayleigh", "love"], "c_tol_rel": TOL, "l2": "flushed between steps (256 MiB write)",
                       "parallelism": f"model-sharded x{world}",
                       "scan_launch_shape": {"fp32": list(tuned[True]), "fp64": list(tuned[False]),
                                             "chosen_by": ("engine defaults (--no-autotune)" if args.no_autotune else
                                                           "autotuner on 1,000 of the models, both waves") +
                                                          ": fused-scan warps per CTA, CTAs per SM, FP32 scan form "
                                                          "(0 automatic: split rounds for Rayleigh, fused for Love; "
                                                          "1 fused; 2 split)"}},
            "fp64": {"value": value64, "unit": "roots/s", "ms_per_step": ms64 / args.steps,
                     "fp32_scan_speedup": value / value64,
                     "stage_ms": {("rayleigh" if w == 0 else "love"): stage64[w] for w in (0, 1)}},
            "e2e": {"value": e2e_value, "unit": "roots/s", "h2d_bytes_per_step": 2 * per_wave_in,
                    "d2h_bytes_per_step": 2 * per_wave_out},
            "roofline": {"bound": "fp32-cuda-core",
                         "kernel": "split_eval32_pair: the FP32 Rayleigh evaluations of the split scan, "
                                   "two samples per thread in paired FP32 instructions",
                         "achieved": achieved / 1e12, "peak": peak32 / 1e12, "unit": "TFLOP/s",
                         "frac": achieved / peak32,
                         "traffic": (EVAL_DRAM_BYTES_PER_STEP * eval_steps / eval_launches
                                     if EVAL_DRAM_BYTES_PER_STEP else None),
                         "launches": eval_launches, "ms_per_launch": eval_ms / eval_launches,
                         "flop_per_launch": eval_flops / eval_launches,
                         "algorithmic_flops": "170 per Rayleigh layer step (secular.cuh, FMA = 2) x FP32 layer "
                                              "steps the kernel evaluated (MD200_STAT_SPLIT_EVAL_STEPS), special "
                                              "functions not counted",
                         "traffic_note": "DRAM bytes per evaluated layer step from an ncu capture of every "
                                         "evaluation launch of a 2,000-model run, times this launch's steps; the "
                                         "kernel reads 32-byte sample records and the model tables and is "
                                         "compute-bound",
                         "peak_kind": "measured FMA throughput (md200_measure_peak), not MEASURED_PEAKS.json",
                         "fp64_peak": peak64 / 1e12,
                         "scan_stage": {"achieved": scan_achieved / 1e12, "frac": scan_achieved / peak32,
                                        "ms_per_step": scan_ms,
                                        "note": "the whole FP32 scan stage of both waves (split rounds for "
                                                "Rayleigh, fused kernel for Love), algorithmic flops of the "
                                                "samples the scans consumed"},
                         "stage_ms": {("rayleigh" if w == 0 else "love"): stage[w] for w in (0, 1)}},
            "cpu_baseline": cpu,
            "cpu_baseline_auto": cpu_auto,
            "gpu_launches": launches * args.steps,
            "clocks": clocks.summary(),
            "engine_stats": {"rayleigh": e32_stats[0], "love": e32_stats[1]},
            "parity": parity,
            "reference_cuda": ref_cuda,
            "config2": config2,
            "jacobian": jac,
            "ragged": ragged,
            "reliability": reliability,
            "uniform": uniform,
        }
        print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
