"""The split FP32 scan against the fused one.

The single-precision scan runs either as one fused kernel (a warp scans one trace
from start to end) or as rounds of split kernels over an active set of traces
(positions one warp per trace, FP32 values one thread per sample -- for Rayleigh
one thread per two samples in paired f32x2 instructions --, FP64 re-evaluations
one thread per listed sample, bookkeeping one thread per trace, trough windows and
last cells one warp per request; modisp_b200/csrc/split_scan.cuh).  The paired
Rayleigh evaluation must give each sample the value the fused kernel's single
evaluation gives (both are explicitly rounded, rayleigh_eval32), pairs mixing
propagating, evanescent and water-top lanes included, and every decision follows
the same rule in the same order, so both must return the same brackets -- and therefore identical velocities, group velocities, flags,
levels and counts, bit for bit -- on crustal, low-velocity-layer and water-layer
batches, the reference suite's frozen fixtures, the large uneven workload (whose
deep models outlast the rounds and are finished by the fused kernel), and with
the scan-point cap that sends traces to the fallback.
"""
import numpy as np
import pytest

from conftest import load_golden, GOLDEN

pytestmark = pytest.mark.gpu

FUSED, SPLIT = 1, 2


def solve(batch, periods, nmodes, wave, mode, bounds=None, **opts):
    from modisp_b200 import _native
    h = batch["thickness"]
    o = _native.default_options()
    o.single_precision, o.group_velocity, o.scan_mode = 1, 1, mode
    for k, v in opts.items():
        setattr(o, k, v)
    e = _native.Engine(0, h.shape[0], h.shape[1], periods.size, nmodes, o)
    try:
        out = e.run(h, batch["vp"], batch["vs"], batch["rho"], periods, bounds, 1e-10, 1., wave, group=True,
                    continuity=True)
        out["launches"] = e.kernel_launches()
        out["stage_ms"] = e.stage_times()
        return out
    finally:
        e.close()


def assert_identical(a, b, where):
    for key in ("velocity", "group_velocity"):
        np.testing.assert_array_equal(a[key].view(np.uint64), b[key].view(np.uint64), err_msg=f"{where}: {key}")
    for key in ("flags", "levels", "counts", "group_velocity_flags", "continuity_flags"):
        np.testing.assert_array_equal(a[key], b[key], err_msg=f"{where}: {key}")
    assert a["stats"]["roots"] == b["stats"]["roots"]


@pytest.mark.parametrize("wave", [0, 1])
@pytest.mark.parametrize("lvz", [0.0, 0.5])
def test_split_equals_fused_on_crustal_batches(wave, lvz):
    from modisp_b200 import workloads
    batch = workloads.crustal_batch(600, workloads.SEED + 80 + int(10 * lvz), lvz_fraction=lvz)
    periods = np.geomspace(0.5, 50., 60)
    fused = solve(batch, periods, 5, wave, FUSED)
    split = solve(batch, periods, 5, wave, SPLIT)
    assert split["launches"] > fused["launches"]  # the rounds did run
    assert split["stats"]["split_eval_layer_steps"] > 0 and fused["stats"]["split_eval_layer_steps"] == 0
    assert split["stage_ms"]["scan_eval"] > 0. and fused["stage_ms"]["scan_eval"] == 0.
    assert_identical(split, fused, f"crustal lvz={lvz} wave={wave}")


@pytest.mark.parametrize("name", sorted(p.stem for p in GOLDEN.glob("fixture_0*.npz")))
def test_split_equals_fused_on_frozen_fixtures(name):
    g = load_golden(name)
    wave = 1 if str(g["wave"]) == "love" else 0
    batch = {k: np.atleast_2d(g[k]) for k in ("thickness", "vp", "vs", "rho")}
    bounds = np.atleast_2d(g["search_bounds"])
    args = (batch, g["periods"], int(g["nmodes"]), wave)
    assert_identical(solve(*args, SPLIT, bounds=bounds), solve(*args, FUSED, bounds=bounds), name)


@pytest.mark.parametrize("wave", [0, 1])
def test_split_equals_fused_on_water_models(wave):
    from modisp_b200 import workloads
    batch = workloads.crustal_batch(300, workloads.SEED + 83, lvz_fraction=0.3)
    batch = {k: v.copy() for k, v in batch.items()}
    # a 1-3 km water layer on top of every model
    rng = np.random.default_rng(5)
    batch["thickness"][:, 0] = rng.uniform(1., 3., batch["thickness"].shape[0])
    batch["vp"][:, 0], batch["vs"][:, 0], batch["rho"][:, 0] = 1.5, 0., 1.03
    periods = np.geomspace(1., 40., 40)
    assert_identical(solve(batch, periods, 4, wave, SPLIT), solve(batch, periods, 4, wave, FUSED), f"water {wave}")


@pytest.mark.parametrize("name", ["ref_crustal48_rayleigh", "ref_lvz48_love"])
def test_split_equals_fused_with_the_scan_point_cap(name):
    g = load_golden(name)
    wave = int(g["wave"])
    batch = {k: np.atleast_2d(g[k]) for k in ("thickness", "vp", "vs", "rho")}
    bounds = np.atleast_2d(g["search_bounds"])
    args = (batch, g["periods"], int(g["nmodes"]), wave)
    split = solve(*args, SPLIT, bounds=bounds, scan_points=48)
    fused = solve(*args, FUSED, bounds=bounds, scan_points=48)
    assert (split["flags"] & 8192).any()  # traces did go to the fallback
    assert_identical(split, fused, f"{name} capped")


@pytest.mark.parametrize("wave", [0, 1])
def test_split_equals_fused_on_the_large_uneven_workload(wave):
    from modisp_b200 import _native, workloads
    batch, periods, modes = workloads.gradient_batch(200, seed=workloads.SEED + 84)
    B, L = batch["thickness"].shape
    off = np.zeros(B + 1, np.int32)
    off[1:] = np.cumsum([p.size for p in periods])
    flat = np.concatenate(periods)
    md = np.asarray(modes, np.int32)
    outs = {}
    for mode in (FUSED, SPLIT):
        o = _native.default_options()
        o.single_precision, o.group_velocity, o.scan_mode = 1, 1, mode
        e = _native.Engine(0, B, L, int(np.diff(off).max()), int(md.max()), o)
        try:
            outs[mode] = e.run_ragged(batch["thickness"], batch["vp"], batch["vs"], batch["rho"], off, flat, md,
                                      1e-10, 1., wave, group=True)
        finally:
            e.close()
    a, b = outs[SPLIT], outs[FUSED]
    for key in ("velocity", "group_velocity"):
        np.testing.assert_array_equal(a[key].view(np.uint64), b[key].view(np.uint64), err_msg=key)
    for key in ("flags", "levels", "counts"):
        np.testing.assert_array_equal(a[key], b[key], err_msg=key)


def test_split_equals_fused_beyond_one_active_set():
    """More traces than the active set holds (2^20): the set is refilled from the
    trace list round after round, and the fused kernel finishes whatever the rounds
    leave -- still the fused scan's results bit for bit."""
    from modisp_b200 import workloads
    batch = workloads.crustal_batch(18_000, workloads.SEED + 85, lvz_fraction=0.3)
    periods = np.geomspace(0.5, 50., 60)  # 1,080,000 traces
    split = solve(batch, periods, 5, 0, SPLIT)
    fused = solve(batch, periods, 5, 0, FUSED)
    assert_identical(split, fused, "beyond one active set")
