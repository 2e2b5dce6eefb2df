"""Launch-shape autotuner for the engine.

The fused scan is a persistent kernel whose best CTA shape depends on the model
depth, the period range and the wave: warps per CTA (1, 2 or 4 traces in flight
per CTA) and the number of resident CTAs per SM trade latency hiding against
instruction-cache and register pressure.  The FP32-scan engine also has two
forms of its scan, which put a different number of threads on a trace: the fused
kernel (one warp per trace) and the split rounds (one thread per sample for the
values, one thread per trace for the bookkeeping, one warp per trace for the
positions); the candidates cover both, and the automatic choice (split for
Rayleigh, fused for Love).  ``autotune`` times each candidate on a sample of the
caller's workload (device time of full runs, best of ``repeats``; both waves
when ``wave`` is None), checks that every candidate returns bit-identical
results (neither the launch shape nor the scan form may change a root), and
caches the fastest per device and workload geometry.

The scan-grid density is not searched: 16 points per phase unit is the
smallest density whose root sets matched the reference on the validation
batches; coarser grids were faster but changed root sets, and denser ones only
cost time.
"""
from __future__ import annotations

import json
import os
from pathlib import Path

import numpy as np

from . import _native

# (warps per CTA, CTAs per SM; 0 = as many as registers allow)
# (warps per CTA, CTAs per SM; 0 = as many as registers allow) of the fused scan
SHAPES = ((4, 0), (4, 3), (4, 2), (2, 0), (2, 4), (1, 0))
# scan forms of the FP32-scan engine (md200_options.scan_mode): 0 automatic
# (split rounds for Rayleigh, fused kernel for Love), 1 fused, 2 split
FP32_MODES = (0, 1, 2)


def candidates(single: bool) -> tuple:
    """(warps per CTA, CTAs per SM, scan form) candidates of an engine."""
    modes = FP32_MODES if single else (0,)
    return tuple((w, b, m) for (w, b) in SHAPES for m in modes)


CANDIDATES = candidates(True)


def cache_path() -> Path:
    base = os.environ.get("MODISP_B200_CACHE") or os.path.join(os.path.expanduser("~"), ".cache", "modisp_b200")
    return Path(base) / "autotune.json"


def workload_key(device_name: str, layers: int, periods: int, nmodes: int, wave, single: bool) -> str:
    """Cache key: device and the geometry buckets that move the optimum."""
    lb = 1 << max(0, int(np.ceil(np.log2(max(layers, 1)))))  # layers rounded up to a power of two
    w = "both" if wave is None else wave
    return f"{device_name}|L{lb}|T{periods}|K{nmodes}|wave{w}|{'fp32' if single else 'fp64'}"


def _load(path: Path) -> dict:
    try:
        return json.loads(path.read_text())
    except (OSError, ValueError):
        return {}


def _store(path: Path, table: dict) -> None:
    try:
        path.parent.mkdir(parents=True, exist_ok=True)
        tmp = path.with_suffix(".tmp")
        tmp.write_text(json.dumps(table, indent=1, sort_keys=True))
        os.replace(tmp, path)
    except OSError:
        pass  # a read-only home only loses the cache


def apply(options, shape) -> None:
    options.warps_per_block, options.blocks_per_sm = int(shape[0]), int(shape[1])
    if len(shape) > 2:
        options.scan_mode = int(shape[2])


def measure(shape, sample, periods, nmodes, wave, single, device=0, repeats=2, tol=1e-10):
    """Device milliseconds of one full run (best of ``repeats``; with wave None the
    sum over both waves) and its outputs (a list, one per wave run)."""
    B, L = sample["thickness"].shape
    o = _native.default_options()
    o.single_precision = int(single)
    o.group_velocity = 1
    apply(o, shape)
    eng = _native.Engine(device, B, L, len(periods), nmodes, o)
    try:
        total, outs = 0., []
        for w in ((0, 1) if wave is None else (wave,)):
            args = (sample["thickness"], sample["vp"], sample["vs"], sample["rho"], np.asarray(periods, float), None,
                    tol, 1., w)
            eng.run(*args, group=True)  # warm-up
            best, out = np.inf, None
            for _ in range(repeats):
                out = eng.run(*args, group=True)
                stages = eng.stage_times()
                stages.pop("scan_eval", None)  # a part of the scan stage, not a stage of its own
                best = min(best, sum(stages.values()))
            total += best
            outs.append(out)
        return total, outs
    finally:
        eng.close()


def autotune(sample, periods, nmodes=5, wave=0, single=True, device=0, candidates=None, use_cache=True,
             timer=measure):
    """Fastest candidate for this workload: (warps_per_block, blocks_per_sm,
    scan_mode).

    ``sample``: a representative [B, L] batch (a few hundred to a few thousand
    models); ``wave``: 0, 1, or None for both waves.  ``candidates`` defaults to
    ``candidates(single)``.  ``timer`` is the measuring function (replaceable in
    tests).
    """
    if candidates is None:
        candidates = globals()["candidates"](single)
    name = _native.device_name(device) if timer is measure else "test-device"
    key = workload_key(name, sample["thickness"].shape[1], len(periods), nmodes, wave, single)
    path = cache_path()
    table = _load(path) if use_cache else {}
    if key in table:
        return tuple(table[key]["shape"])
    results, reference = [], None
    for shape in candidates:
        ms, out = timer(shape, sample, periods, nmodes, wave, single, device)
        outs = out if isinstance(out, list) else [out]
        if reference is None:
            reference = outs
        elif out is not None:
            for a, b in zip(outs, reference):
                for field in ("velocity", "counts", "flags"):
                    if not np.array_equal(np.asarray(a[field]).view(np.uint8), np.asarray(b[field]).view(np.uint8)):
                        raise RuntimeError(f"candidate {shape} changed the {field} output")
        results.append((ms, tuple(shape)))
    ms, shape = min(results)
    if use_cache:
        table[key] = {"shape": list(shape), "ms": ms,
                      "timings": {"x".join(str(v) for v in s): t for t, s in results}}
        _store(path, table)
    return tuple(shape)
