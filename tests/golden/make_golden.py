"""Generate the golden fixtures under tests/golden/ from the reference implementation.

Run with the reference CPU engine built by ``make -C oracle`` and, for the
repacked frozen fixtures and the reliability cases, the path of a reference
source checkout:

    python tests/golden/make_golden.py --reference <modisp checkout>
    python tests/golden/make_golden.py --only deep     # no checkout needed

Outputs (all small .npz files, committed):

* ``ref_<case>.npz``: inputs and the reference CPU engine's outputs with the
  parity settings (accuracy high, shape-adaptive search, Dunkin secular, Brent
  refinement, Love phase strategy, c_tol_rel 1e-12, group velocity at the
  default group_rtol 1e-3).  Cases: the quickstart model (Rayleigh, Love),
  48-model subsets of the crustal batch (Rayleigh, Love), 48 low-velocity-layer
  models (Rayleigh, Love), six surface-water models (Rayleigh), four deep
  slow-over-fast models at 63, 100 and 256 modes (Rayleigh, Love; their short
  periods hold more roots than the guard-extended mode count), one crustal model
  with a close pair whose shape-feature trough lies in the FP32 scan's FP64 band, and
  one low-velocity-layer model with a pair in the last cell before the cutoff.
* ``jac_<case>.npz``: phase-velocity Jacobians by central differences (step 1e-6
  relative) of the reference CPU solver's roots (c_tol_rel 1e-13): four
  config-4 models (Rayleigh), two (Love), two surface-water models (Rayleigh).
* ``fixture_<name>.npz``: the reference test suite's own frozen fixtures
  (tests/data/accuracy_high_cpu_linux/*.npz, tests/data/witness_*.npz,
  tests/data/B10000_*.npz) repacked with their inputs and expected roots.
* ``reliability_<case>.npz``: inputs and outputs of the reference's cross-period
  mode-reliability checks (python/modisp/reliability.py, loaded from its file):
  the cases of the reference's own tests, seeded synthetic batches (unsorted and
  duplicate periods, gaps, NaNs, crossing ranks, failure and uncertainty bits,
  negative counts, every option non-default) and two reference-solver results.
  ``--only reliability`` regenerates just these.
"""
from __future__ import annotations

import argparse
import importlib.util
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from modisp_b200 import workloads  # noqa: E402

FIELDS = ("phase_velocity", "trace_flags", "search_level", "root_count", "search_bounds",
          "group_velocity", "group_velocity_flags")


def save_reference_case(name, batch, periods, nmodes, wave):
    out = oracle.reference_solve(batch["thickness"], batch["vp"], batch["vs"], batch["rho"], periods,
                                 nmodes, wave=wave, tol=1e-12, group_velocity=True, group_rtol=1e-3)
    np.savez_compressed(HERE / f"ref_{name}.npz", thickness=np.atleast_2d(batch["thickness"]),
                        vp=np.atleast_2d(batch["vp"]), vs=np.atleast_2d(batch["vs"]),
                        rho=np.atleast_2d(batch["rho"]), periods=periods, nmodes=nmodes, wave=wave,
                        tol=1e-12, **{k: out[k] for k in FIELDS})
    valid = int(np.isfinite(out["phase_velocity"]).sum())
    print(f"ref_{name}: {valid} valid roots")


def subset(batch, idx):
    return {k: v[idx] for k, v in batch.items()}


def water_models():
    rng = np.random.default_rng(workloads.SEED + 7)
    rows = []
    for _ in range(6):
        n = int(rng.integers(3, 7))
        vs = np.sort(rng.uniform(0.4, 3.6, n + 1))
        vp = vs * rng.uniform(1.7, 2.0, n + 1)
        h = rng.uniform(0.2, 2.0, n + 1)
        h[-1] = 0.
        vs = np.concatenate([[0.], vs])
        vp = np.concatenate([[1.5], vp])
        h = np.concatenate([[rng.uniform(0.01, 0.5)], h])
        rho = np.concatenate([[1.02], 1.74 * vp[1:] ** 0.25])
        rows.append((h, vp, vs, rho))
    return workloads._pad(rows, max(r[0].size for r in rows))


def save_jacobian_case(name, batch, periods, nmodes, wave):
    """Central differences of the reference solver's roots (the phase-velocity
    Jacobian the engine's adjoint must reproduce)."""
    B, L = batch["thickness"].shape
    roots = np.full((B, nmodes, len(periods)), np.nan)
    jac = np.zeros((B, nmodes, len(periods), 4, L))
    for b in range(B):
        roots[b], jac[b] = oracle.reference_fd_phase_jacobian(
            batch["thickness"][b], batch["vp"][b], batch["vs"][b], batch["rho"][b], periods, nmodes, wave)
    np.savez_compressed(HERE / f"jac_{name}.npz", thickness=batch["thickness"], vp=batch["vp"], vs=batch["vs"],
                        rho=batch["rho"], periods=periods, nmodes=nmodes, wave=wave, rel_step=1e-6, tol=1e-13,
                        phase_velocity=roots, jac_phase_fd=jac)
    print(f"jac_{name}: {int(np.isfinite(roots).sum())} roots")


def repack_reference_fixtures(reference: Path):
    data = reference / "tests" / "data"
    for path in sorted((data / "accuracy_high_cpu_linux").glob("*.npz")):
        f = np.load(path, allow_pickle=True)
        keep = {k: np.asarray(f[k]) for k in ("thickness", "vp", "vs", "rho", "periods", "nmodes", "cmin",
                                               "cmax", "phase_velocity", "mode_mask", "root_count",
                                               "search_bounds", "trace_flags")}
        keep["wave"] = np.asarray(str(f["wave"]))
        np.savez_compressed(HERE / f"fixture_{path.stem}.npz", **keep)
        print("fixture", path.stem)
    for path in sorted(data.glob("witness_*.npz")) + sorted(data.glob("B10000_*.npz")):
        f = np.load(path)
        keep = {k: np.asarray(f[k]) for k in f.files}
        np.savez_compressed(HERE / f"fixture_{path.stem}.npz", **keep)
        print("fixture", path.stem)


def load_reference_reliability(reference: Path):
    spec = importlib.util.spec_from_file_location("reference_reliability",
                                                  reference / "python" / "modisp" / "reliability.py")
    module = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(module)
    return module


def synthetic_reliability(seed, B, K, T, duplicates=True, gaps=True):
    """Mode curves with the defects the checks look for, in shuffled period order."""
    rng = np.random.default_rng(seed)
    p = np.sort(np.exp(rng.uniform(np.log(.5), np.log(50.), T)))
    if gaps:
        p[T // 2:] *= np.exp(.6)  # one gap above the default 0.25 log units
    if duplicates:
        p[3] = p[2]
        p[T - 2] = p[T - 3]
    base = 1. + np.arange(K)[None, :, None] * (.35 + .1 * rng.random((B, 1, 1)))
    v = base * (1. + .25 * np.log(p)[None, None, :] / np.log(50.)) + 1e-3 * rng.standard_normal((B, K, T))
    v[rng.random(v.shape) < .01] = np.nan  # holes
    hi = rng.random((B, T)) < .03  # lost top modes
    v[:, -1, :][hi] = np.nan
    if K >= 2:
        swap = rng.random((B, T)) < .03  # crossing ranks
        v[:, [0, 1], :] = np.where(swap[:, None, :], v[:, [1, 0], :], v[:, [0, 1], :])
    if K >= 3:
        close = rng.random((B, T)) < .03  # near-degenerate pairs
        v[:, 2, :] = np.where(close, v[:, 1, :] * (1. + 1e-3), v[:, 2, :])
    jump = rng.random((B, K, T)) < .02  # step jumps
    v = np.where(jump, v * 1.3, v)
    if duplicates:
        dup_noise = rng.random((B, K)) < .2  # duplicates that disagree
        v[:, :, 3] = np.where(dup_noise, v[:, :, 2] * (1. + 1e-6), v[:, :, 2])
    order = rng.permutation(T)
    tf = (rng.integers(0, 2, (B, T)) * rng.choice([1, 2, 4, 8, 2048, 4096, 1 << 20], (B, T))).astype(np.uint32)
    tf[rng.random((B, T)) < .7] = 0
    counts = np.isfinite(v).sum(axis=1).astype(np.int32)
    counts[rng.random((B, T)) < .03] = -1
    counts[rng.random((B, T)) < .03] += 1
    return v[:, :, order], p[order], tf[:, order], counts[:, order]


def save_reliability_case(rel, name, velocity, periods, trace_flags=None, root_count=None, **options):
    r = rel.check_mode_reliability(velocity, periods, trace_flags=trace_flags, root_count=root_count, **options)
    extra = {}
    if trace_flags is not None:
        extra["trace_flags"] = np.asarray(trace_flags)
    if root_count is not None:
        extra["root_count"] = np.asarray(root_count)
    np.savez_compressed(HERE / f"reliability_{name}.npz", velocity=np.asarray(velocity, float),
                        periods=np.asarray(periods, float), flags=r.flags, assessed=r.assessed,
                        previous_index=r.previous_index, sorted_order=r.sorted_order,
                        options=np.array([options.get(k, d) for k, d in RELIABILITY_DEFAULTS]), **extra)
    print(f"reliability_{name}: {int((r.flags != 0).sum())} flagged of {r.flags.size}")


# option names and the reference's defaults, in the order stored in the fixtures
RELIABILITY_DEFAULTS = (("close_root_rtol", .005), ("max_relative_step", .1), ("prediction_rtol", .05),
                        ("max_log_period_gap", .25))


def save_reliability_cases(reference: Path):
    rel = load_reference_reliability(reference)
    # the reference test suite's cases (tests/test_reliability.py)
    save_reliability_case(rel, "sort_dup_gap", np.array([[[1.02, 1., 1.01, 1.01, 1.2], [2.02, 2., 2.01, 2.01, 2.2]]]),
                          np.array([1.2, 1., 1.1, 1.1, 4.]))
    bad = np.array([[[1.02, 1., 1.01, 1.01 + 1e-4, 1.2], [2.02, 2., 2.01, 2.01, 2.2]]])
    save_reliability_case(rel, "dup_mismatch", bad, np.array([1.2, 1., 1.1, 1.1, 4.]))
    save_reliability_case(rel, "birth_rank_failure", np.array([[[1., 1.3, 1.8], [1.4, 1.8, np.nan], [2., 2.05, 2.1]]]),
                          np.array([1., 1.1, 1.2]), trace_flags=np.array([[0, 4096, 4]], dtype=np.uint32))
    p = np.array([1e100, np.nextafter(1e100, np.inf), np.nextafter(np.nextafter(1e100, np.inf), np.inf)])
    save_reliability_case(rel, "adjacent_periods", np.ones((1, 1, 3)), p)
    # seeded synthetic batches
    v, p, tf, counts = synthetic_reliability(workloads.SEED + 21, 40, 6, 25)
    save_reliability_case(rel, "synthetic_full", v, p, trace_flags=tf, root_count=counts)
    save_reliability_case(rel, "synthetic_plain", v, p)
    save_reliability_case(rel, "synthetic_options", v, p, trace_flags=tf, root_count=counts, close_root_rtol=.02,
                          max_relative_step=.03, prediction_rtol=.01, max_log_period_gap=.5)
    v1, p1, tf1, c1 = synthetic_reliability(workloads.SEED + 22, 7, 1, 9, duplicates=False)
    save_reliability_case(rel, "single_mode", v1, p1, trace_flags=tf1, root_count=c1)
    save_reliability_case(rel, "single_period", v[:, :, :1], p[:1], trace_flags=tf[:, :1], root_count=counts[:, :1])
    # reference-solver results
    for case in ("lvz48_rayleigh", "crustal48_love"):
        f = np.load(HERE / f"ref_{case}.npz")
        save_reliability_case(rel, case, f["phase_velocity"], f["periods"], trace_flags=f["trace_flags"],
                              root_count=f["root_count"])


def save_deep_cases():
    """Deep models at mode counts far above the usual five (63, 100 and 256)."""
    deep = workloads.deep_batch(4)
    periods = np.geomspace(0.5, 20., 8)
    for nmodes in (63, 100, 256):
        for wave, name in ((0, "rayleigh"), (1, "love")):
            save_reference_case(f"deep4_k{nmodes}_{name}", deep, periods, nmodes, wave)


def reference_tree(args):
    if not args.reference:
        raise SystemExit("pass --reference <modisp source checkout> (frozen fixtures and reliability cases)")
    return Path(args.reference)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", help="path of the reference (modisp) source checkout")
    ap.add_argument("--only", choices=["reliability", "deep"])
    args = ap.parse_args()
    if args.only == "reliability":
        save_reliability_cases(reference_tree(args))
        return
    if oracle.reference() is None:
        raise SystemExit("build the reference CPU engine first: make -C oracle")
    if args.only == "deep":
        save_deep_cases()
        return
    tree = reference_tree(args)
    model, periods = workloads.quickstart()
    save_reference_case("quickstart_rayleigh", model, periods, 2, 0)
    save_reference_case("quickstart_love", model, periods, 2, 1)
    batch, periods, nmodes = workloads.config2(10_000)
    idx = np.arange(0, 10_000, 10_000 // 48)[:48]
    save_reference_case("crustal48_rayleigh", subset(batch, idx), periods, nmodes, 0)
    save_reference_case("crustal48_love", subset(batch, idx), periods, nmodes, 1)
    lvz = workloads.crustal_batch(400, workloads.SEED + 3, lvz_fraction=1.0)
    save_reference_case("lvz48_rayleigh", subset(lvz, np.arange(48)), periods, nmodes, 0)
    save_reference_case("lvz48_love", subset(lvz, np.arange(48)), periods, nmodes, 1)
    save_reference_case("water6_rayleigh", water_models(), np.geomspace(0.2, 20., 24), 4, 0)
    # a close pair (2.6293 / 2.6359 km/s at T = 9.7 s) whose trough floor lies in the
    # band the FP32 scan re-evaluates in FP64
    pair = workloads.crustal_batch(2000, workloads.SEED + 2)
    save_reference_case("pair1678_rayleigh", subset(pair, np.arange(1678, 1679)), periods, nmodes, 0)
    # a low-velocity-layer model with a pair (4.1023 / 4.1185 km/s at T = 13.3 s) in the
    # last grid cell before the half-space cutoff
    lvz5k = workloads.crustal_batch(5000, workloads.SEED + 3, lvz_fraction=0.3)
    save_reference_case("pair3501_rayleigh", subset(lvz5k, np.arange(3501, 3502)), periods, nmodes, 0)
    c4, periods4, nmodes4 = workloads.config4(16)
    save_jacobian_case("config4_rayleigh", subset(c4, np.arange(4)), periods4, nmodes4, 0)
    save_jacobian_case("config4_love", subset(c4, np.arange(4, 6)), periods4, nmodes4, 1)
    save_jacobian_case("water_rayleigh", subset(water_models(), np.arange(2)), np.geomspace(0.5, 20., 12), 3, 0)
    save_deep_cases()
    repack_reference_fixtures(tree)
    save_reliability_cases(tree)


if __name__ == "__main__":
    main()
