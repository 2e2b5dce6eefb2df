"""Generate the golden fixtures under tests/golden/ from the reference implementation.

Run in a checkout that has the reference source tree (default /root/reference)
and the reference CPU engine built by ``make -C oracle``:

    python tests/golden/make_golden.py [--reference /root/reference]

Outputs (all small .npz files, committed):

* ``ref_<case>.npz``: inputs and the reference CPU engine's outputs with the
  parity settings (accuracy high, shape-adaptive search, Dunkin secular, Brent
  refinement, Love phase strategy, c_tol_rel 1e-12, group velocity at the
  default group_rtol 1e-3).  Cases: the quickstart model (Rayleigh, Love),
  48-model subsets of the crustal batch (Rayleigh, Love), 48 low-velocity-layer
  models (Rayleigh, Love), six surface-water models (Rayleigh), one crustal model
  with a close pair whose shape-feature trough lies in the FP32 scan's FP64 band, and
  one low-velocity-layer model with a pair in the last cell before the cutoff.
* ``jac_<case>.npz``: phase-velocity Jacobians by central differences (step 1e-6
  relative) of the reference CPU solver's roots (c_tol_rel 1e-13): four
  config-4 models (Rayleigh), two (Love), two surface-water models (Rayleigh).
* ``fixture_<name>.npz``: the reference test suite's own frozen fixtures
  (tests/data/accuracy_high_cpu_linux/*.npz, tests/data/witness_*.npz,
  tests/data/B10000_*.npz) repacked with their inputs and expected roots.
"""
from __future__ import annotations

import argparse
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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    args = ap.parse_args()
    if oracle.reference() is None:
        raise SystemExit("build the reference CPU engine first: make -C oracle")
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
    repack_reference_fixtures(Path(args.reference))


if __name__ == "__main__":
    main()
