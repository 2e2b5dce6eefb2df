"""The whole 1,000,000-model ragged workload, checked through properties that hold at
any size.

    python tests/full_config5.py            # on a machine with the GPU

Smooth-gradient models of 30-100 thin layers, each with its own 50-120 periods in
0.2-100 s and 1-10 modes, Rayleigh and Love, FP32 scan / FP64 refinement, group
velocities, run as ragged batches of 65,536 models (``dispersion_ragged``).  For
every trace: no unconverged search, roots ascending with the mode index, and the
finite roots exactly the first min(root count, modes) slots.  On the first chunk
the FP32-scan and plain FP64 engines must also agree (masks, counts, phase and
group velocity to 1e-9).  Prints one JSON summary.  Not collected by pytest; the
per-model reference parity of this workload is tests/test_ragged_gpu.py.
"""
import json
import sys
import time
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))

from modisp_b200 import workloads  # noqa: E402
from modisp_b200.ragged import dispersion_ragged  # noqa: E402

MODELS = 1_000_000
CHUNK = 65_536


def check_chunk(res):
    """(roots, unconverged traces, order violations, mask/count violations) of one result."""
    T = np.diff(res.period_offsets)
    modes = res.modes
    cells = modes * T
    v = res.phase_velocity
    # per cell: its model's period count and its mode index
    Tc = np.repeat(T, cells)
    start = np.repeat(res.out_offsets, cells)
    idx = np.arange(v.size)
    mode = (idx - start) // np.maximum(Tc, 1)
    last = np.repeat(modes, cells) - 1
    succ = np.where(mode < last, idx + Tc, idx)
    both = np.isfinite(v) & np.isfinite(v[succ]) & (succ != idx)
    order_bad = int(np.count_nonzero(both & ~(v[succ] > v)))
    # finite roots per trace are the first min(count, modes) slots
    tr_of_cell = np.repeat(res.period_offsets[:-1], cells) + (idx - start) % np.maximum(Tc, 1)
    finite_per_trace = np.bincount(tr_of_cell, weights=np.isfinite(v), minlength=res.root_count.size).astype(int)
    expect = np.minimum(np.maximum(res.root_count, 0), np.repeat(modes, T))
    prefix_bad = int(np.count_nonzero(finite_per_trace != expect))
    # a finite root never follows a missing one within a trace
    hole = ~np.isfinite(v) & np.isfinite(v[succ]) & (succ != idx)
    prefix_bad += int(np.count_nonzero(hole))
    unconverged = int(np.count_nonzero(res.trace_flags & 4))
    return int(np.isfinite(v).sum()), unconverged, order_bad, prefix_bad


def main():
    t0 = time.time()
    batch, periods, modes = workloads.gradient_batch(MODELS, seed=workloads.SEED + 50)
    gen_s = time.time() - t0
    summary = {"models": MODELS, "traces": int(sum(p.size for p in periods)),
               "cells": int(sum(p.size * m for p, m in zip(periods, modes))), "generate_s": round(gen_s, 1)}
    for wave in ("rayleigh", "love"):
        tot = dict(roots=0, unconverged_traces=0, order_violations=0, mask_count_violations=0)
        t1 = time.time()
        for s in range(0, MODELS, CHUNK):
            e = min(MODELS, s + CHUNK)
            sub = {k: batch[k][s:e] for k in batch}
            res = dispersion_ragged(sub["thickness"], sub["vp"], sub["vs"], sub["rho"], periods[s:e],
                                    nmodes=np.asarray(modes[s:e]), wave=wave, precision="mixed",
                                    group_velocity=True, chunk_models=CHUNK)
            r, u, o, p = check_chunk(res)
            tot["roots"] += r
            tot["unconverged_traces"] += u
            tot["order_violations"] += o
            tot["mask_count_violations"] += p
            if s == 0:
                ref = dispersion_ragged(sub["thickness"], sub["vp"], sub["vs"], sub["rho"], periods[s:e],
                                        nmodes=np.asarray(modes[s:e]), wave=wave, precision="float64",
                                        group_velocity=True, chunk_models=CHUNK)
                a, b = res.phase_velocity, ref.phase_velocity
                m = np.isfinite(b)
                g = np.isfinite(res.group_velocity) & np.isfinite(ref.group_velocity)
                tot["first_chunk_fp32_vs_fp64"] = dict(
                    models=e - s, mask_mismatches=int(np.count_nonzero(np.isfinite(a) != m)),
                    count_mismatches=int(np.count_nonzero(res.root_count != ref.root_count)),
                    max_rel_phase=float(np.max(np.abs(a[m] - b[m]) / b[m])),
                    max_rel_group=float(np.max(np.abs(res.group_velocity[g] - ref.group_velocity[g]) /
                                               ref.group_velocity[g])))
        tot["seconds"] = round(time.time() - t1, 1)
        summary[wave] = tot
        print(wave, tot, flush=True)
    print(json.dumps(summary))


if __name__ == "__main__":
    main()
