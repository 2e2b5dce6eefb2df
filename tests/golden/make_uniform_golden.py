"""Generate tests/golden/uniform_<case>.npz from the reference's own legacy uniform path.

The reference serves search_strategy="uniform" only on CUDA (cpp/cuda/coarse_scan.cu,
cpp/cuda/refine.cu, bound as CoarseScan / Refine in cpp/cuda/bindings.cpp:121-345).
This script drives that extension, compiled for sm_100a by
``make -C oracle REFERENCE=<checkout> ref-cuda`` (oracle/_ref/cuda/_cuda*.so), so it
needs a GPU; it reads nothing else of the reference.  Run it on a B200 from the
repository root:

    python tests/golden/make_uniform_golden.py [--out tests/golden]

Each file holds the inputs (thickness, vp, vs, rho, periods, nmodes, nc, cmin,
cmax, c_tol_rel, f_accept), the reference's stage 1 values (``rows``, float32
[B, T, nc]) and its stage 2 outputs (``phase_velocity`` [B, nmodes, T],
``trace_flags`` [B, T], ``stats`` in STAT_NAMES order).  Cases (all solid,
Rayleigh, seeded workloads of modisp_b200.workloads):

* crustal12 -- 12 crustal models, 10 periods 0.5-50 s, 5 modes, nc 512, cmin 0.2;
* lvz12     -- 12 models with a low-velocity layer, 10 periods 1-40 s, 6 modes,
               nc 256, f_accept 0.3 (roots screened by |F|);
* lowc6     -- 6 crustal models scanned from cmin 0.02, where single-precision
               values of the deepest layers lose their sign (rejected and
               relocated brackets);
* deep4     -- 4 deep slow-over-fast models, 6 periods 0.5-16 s, 40 modes, nc 1024
               (more modes than a warp has lanes).
"""
from __future__ import annotations

import argparse
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))


def cases():
    from modisp_b200 import workloads as w
    crustal, _, _ = w.config2(10_000)
    pick = lambda batch, idx: {k: np.ascontiguousarray(v[idx]) for k, v in batch.items()}  # noqa: E731
    return {
        "crustal12": (pick(crustal, np.arange(12) * 811), np.geomspace(0.5, 50., 10), 5, 512, 0.2, 1.0),
        "lvz12": (w.crustal_batch(12, w.SEED + 7, lvz_fraction=1.0), np.geomspace(1., 40., 10), 6, 256, 0.2, 0.3),
        "lowc6": (pick(crustal, np.arange(6) * 1301 + 5), np.geomspace(0.5, 30., 8), 4, 512, 0.02, 1.0),
        "deep4": (w.deep_batch(4, w.SEED + 8), np.geomspace(0.5, 16., 6), 40, 1024, 0.2, 1.0),
    }


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--out", default=str(ROOT / "tests" / "golden"))
    args = ap.parse_args(argv)
    import oracle
    ref = oracle.reference_cuda()
    if ref is None:
        raise SystemExit("the reference CUDA extension is not built (make -C oracle REFERENCE=<checkout> ref-cuda)")
    out = Path(args.out)
    out.mkdir(parents=True, exist_ok=True)
    c_tol_rel = 1e-6
    for name, (batch, periods, nmodes, nc, cmin, f_accept) in cases().items():
        h, vp, vs, rho = (np.ascontiguousarray(batch[k], dtype=np.float64) for k in ("thickness", "vp", "vs", "rho"))
        B, L = h.shape
        cmax = float(vs[:, -1].max())  # the legacy solver's default (python/modisp/_legacy.py:275-279)
        scan = ref.CoarseScan(B, L)
        scan.upload_models(h, vp, vs, rho)
        scan.upload_periods(periods)
        scan.allocate(nc)
        rows = scan.scan(cmin, cmax)
        refine = ref.Refine(B, L)
        refine.upload_models(h, vp, vs, rho)
        refine.upload_periods(periods)
        refine.allocate(nc, nmodes)
        refine.run(scan, cmin, cmax, c_tol_rel, f_accept, nmodes)
        velocity, flags, stats = refine.download(), refine.flags(), refine.stats()
        np.savez_compressed(out / f"uniform_{name}.npz", thickness=h, vp=vp, vs=vs, rho=rho, periods=periods,
                            nmodes=nmodes, nc=nc, cmin=cmin, cmax=cmax, c_tol_rel=c_tol_rel, f_accept=f_accept,
                            rows=rows, phase_velocity=velocity, trace_flags=flags,
                            stats=np.array([stats[k] for k in ref.STAT_NAMES], np.uint64),
                            stat_names=np.array(ref.STAT_NAMES))
        print(name, B, L, "roots", int(np.isfinite(velocity).sum()), stats)


if __name__ == "__main__":
    main()
