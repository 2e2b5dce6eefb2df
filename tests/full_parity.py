"""Full-batch parity of both engines against the reference CPU engine.

    python tests/full_parity.py            # on a machine with the GPU and oracle/_ref built

Solves the whole 10,000-model crustal batch (60 periods, 5 modes, both waves) with
the reference CPU engine (tol 1e-12, all host cores) and with the FP32-scan and
FP64 engines, and reports per engine and wave: traces whose mode masks differ,
root-count mismatches, the largest relative phase difference, and the largest
relative group-velocity difference from the oracle's long-double value on 400
random roots.  Not collected by pytest (it takes a few minutes of CPU); the fast
parity tests are tests/test_parity_gpu.py.
"""
import json
import os
import sys
import time
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
import numpy as np
import oracle
from modisp_b200 import _native, workloads
batch, periods, nmodes = workloads.config2()
B, L = batch["thickness"].shape
T = periods.size
threads = len(os.sched_getaffinity(0))
res = {"models": B, "periods": T, "nmodes": nmodes, "threads": threads}
rng = np.random.default_rng(7)
for wave, name in ((0, "rayleigh"), (1, "love")):
    t0 = time.time()
    ref = oracle.reference_solve(batch["thickness"], batch["vp"], batch["vs"], batch["rho"], periods, nmodes,
                                 wave=wave, tol=1e-12, threads=threads)
    tref = time.time() - t0
    rv = ref["phase_velocity"]
    for single in (1, 0):
        o = _native.default_options(); o.single_precision = single; o.group_velocity = 1
        e = _native.Engine(0, B, L, T, nmodes, o)
        out = e.run(batch["thickness"], batch["vp"], batch["vs"], batch["rho"], periods, None, 1e-10, 1., wave, group=True)
        e.close()
        v = out["velocity"]
        fm = np.isfinite(v); rm = np.isfinite(rv)
        both = fm & rm
        mask_mm = int(np.any(fm != rm, axis=1).sum())
        cnt_mm = int((out["counts"] != ref["root_count"]).sum())
        ph = float((np.abs(v[both] - rv[both]) / rv[both]).max())
        # group velocity against the oracle's long-double value on a random sample of roots
        cells = np.argwhere(both)
        pick = cells[rng.choice(len(cells), 400, replace=False)]
        gerr = 0.
        for b, k, f in pick:
            c = v[b, k, f]
            u = oracle.group(batch["thickness"][b], batch["vp"][b], batch["vs"][b], batch["rho"][b], periods[f], c,
                             c * (1 - 1e-6), c * (1 + 1e-6), wave)
            g = out["group_velocity"][b, k, f]
            if np.isfinite(u) and np.isfinite(g):
                gerr = max(gerr, abs(g - u) / u)
        key = f"{name}_{'fp32scan' if single else 'fp64'}"
        res[key] = dict(roots=int(both.sum()), mask_mismatch_traces=mask_mm, count_mismatches=cnt_mm,
                        max_rel_phase=ph, max_rel_group_vs_oracle_400=gerr)
        print(key, res[key], flush=True)
    res[f"{name}_reference_seconds"] = tref
print(json.dumps(res))
