"""The engine as a drop-in for modisp's CUDA backend, driven by the reference's own
unmodified Python wrapper.

The oracle recipe (``make -C oracle REFERENCE=<checkout>``) stages the reference's
``python/modisp`` package, unmodified, into ``oracle/_ref/modisp`` with the
reference CPU engine as its ``_cpu`` module.  Imported from there, its loader
(python/modisp/_loader.py:15-28) finds this repository's ``modisp_cuda`` package
and ``Solver._solve``'s chunk loop (python/modisp/__init__.py:379-444) drives the
plugin's ``QeSolver``.  Each result is compared with the same wrapper's
``backend="cpu"`` on the same inputs: mode masks and root counts identical, phase
velocities within 1e-9 (FP64 output) or the float32 output's rounding.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12
THREADS = min(256, len(os.sched_getaffinity(0)))


@pytest.fixture(scope="module")
def modisp():
    import oracle
    wrapper = oracle.reference_wrapper()
    if wrapper is None:
        pytest.skip("reference wrapper not staged (make -C oracle REFERENCE=<checkout>)")
    return wrapper


def solve(modisp, batch, periods, nmodes, wave, **options):
    return modisp.dispersion_batch(batch["thickness"], batch["vp"], batch["vs"], batch["rho"], periods,
                                   nmodes=nmodes, wave=wave, **options)


def compare(cuda, cpu, rtol):
    assert cuda.backend_used == "cuda" and cpu.backend_used == "cpu"
    np.testing.assert_array_equal(cuda.mode_mask, cpu.mode_mask)
    np.testing.assert_array_equal(cuda.root_count, cpu.root_count)
    m = cpu.mode_mask
    rel = np.abs(cuda.phase_velocity[m].astype(np.float64) - cpu.phase_velocity[m]) / cpu.phase_velocity[m]
    assert rel.max(initial=0.) <= rtol, f"max |dc|/c {rel.max():.3e}"
    return rel.max(initial=0.)


def crustal64():
    from modisp_b200 import workloads
    batch, periods, nmodes = workloads.config2(10_000)
    idx = np.arange(64) * 150
    return {k: v[idx] for k, v in batch.items()}, periods, nmodes


@pytest.mark.parametrize("wave", ["rayleigh", "love"])
def test_quickstart_through_the_reference_wrapper(modisp, wave):
    from modisp_b200 import workloads
    model, periods = workloads.quickstart()
    batch = {k: v[None] for k, v in model.items()}
    opts = dict(accuracy="high", c_tol_rel=TOL, group_velocity=True)
    cuda = solve(modisp, batch, periods, 2, wave, backend="cuda", **opts)
    cpu = solve(modisp, batch, periods, 2, wave, backend="cpu", threads=THREADS, **opts)
    compare(cuda, cpu, 1e-9)
    # structural group-velocity flags (missing root, close root) agree
    for bit in (1, 16):
        np.testing.assert_array_equal(cuda.group_velocity_flags & bit, cpu.group_velocity_flags & bit)


@pytest.mark.parametrize("wave", ["rayleigh", "love"])
def test_crustal_batch_through_the_reference_wrapper(modisp, wave):
    batch, periods, nmodes = crustal64()
    opts = dict(accuracy="high", c_tol_rel=TOL, group_velocity=True)
    cuda = solve(modisp, batch, periods, nmodes, wave, backend="cuda", **opts)
    cpu = solve(modisp, batch, periods, nmodes, wave, backend="cpu", threads=THREADS, **opts)
    compare(cuda, cpu, 1e-9)
    for bit in (1, 16):
        np.testing.assert_array_equal(cuda.group_velocity_flags & bit, cpu.group_velocity_flags & bit)


@pytest.mark.parametrize("wave", ["rayleigh", "love"])
def test_float32_precision_with_canonical_lower_bound(modisp, wave):
    """precision="float32" with the default cmin: the wrapper passes canonical_lower
    (python/modisp/__init__.py:411-422) and receives float32 phase velocities."""
    batch, periods, nmodes = crustal64()
    cuda = solve(modisp, batch, periods, nmodes, wave, backend="cuda", accuracy="high", c_tol_rel=TOL,
                 precision="float32")
    cpu = solve(modisp, batch, periods, nmodes, wave, backend="cpu", threads=THREADS, accuracy="high",
                c_tol_rel=TOL)
    assert cuda.phase_velocity.dtype == np.float32
    compare(cuda, cpu, 2. ** -23 + 1e-9)  # float32 rounding of an FP64-refined root


@pytest.mark.parametrize("wave", ["rayleigh", "love"])
def test_default_auto_preset_with_continuity_check(modisp, wave):
    """The reference's default accuracy ("auto") with its continuity screen on: the
    wrapper screens the plugin's output with its own _cpu.continuity_screen and
    reviews suspects through the plugin.  The engine searches exhaustively at
    every preset, so its roots match the CPU engine at accuracy="high"."""
    batch, periods, nmodes = crustal64()
    cuda = solve(modisp, batch, periods, nmodes, wave, backend="cuda", group_velocity=True, continuity_check=True)
    assert cuda.accuracy == "auto"
    cpu = solve(modisp, batch, periods, nmodes, wave, backend="cpu", threads=THREADS, accuracy="high",
                c_tol_rel=TOL)
    compare(cuda, cpu, 2e-5)  # the auto preset's c_tol_rel is 1e-5
    assert cuda.continuity_flags is not None


@pytest.mark.parametrize("wave", ["rayleigh", "love"])
def test_continuity_review_repairs_planted_suspects_through_the_plugin(modisp, wave):
    """The wrapper's own FP64 review (python/modisp/_continuity.py:17-205) on suspects
    planted on the host: a nested accuracy="high" Solver re-solves them through the
    plugin (one period per row, SUPPORTS_ROW_PERIODS) and their group velocities come
    from the plugin's _review_groups."""
    from modisp import _continuity
    batch, periods, nmodes = crustal64()
    solver = modisp.Solver(backend="cuda", accuracy="balanced", group_velocity=True, continuity_check=True)
    res = solver(batch["thickness"], batch["vp"], batch["vs"], batch["rho"], periods, nmodes, wave)
    velocity = res.phase_velocity.copy()
    trace, levels, counts = res.trace_flags.copy(), res.search_level.copy(), res.root_count.copy()
    group, gflags = res.group_velocity.copy(), res.group_velocity_flags.copy()
    rng = np.random.default_rng(7)
    B, K, T = velocity.shape
    picks = [(b, f) for b, f in zip(rng.integers(0, B, 40), rng.integers(1, T - 1, 40)) if res.mode_mask[b, 0, f]]
    picks = sorted(set(picks))[:12]
    assert len(picks) >= 6
    flags = np.zeros((B, T), np.uint8)
    for b, f in picks:  # plant a wrong root and mark the trace an envelope suspect
        velocity[b, 0, f] *= 1.07
        group[b, 0, f] = 0.
        flags[b, f] = int(_continuity.ContinuityFlag.ENVELOPE)
    stats = dict(continuity_suspected=0, continuity_local_searches=0, continuity_full_searches=0,
                 continuity_repaired=0, continuity_unresolved=0, continuity_evaluations=0, group_evaluations=0,
                 group_invalid=0, evaluations=0)
    models = tuple(np.ascontiguousarray(batch[k]) for k in ("thickness", "vp", "vs", "rho"))
    _continuity.review(solver, "cuda", models, periods, wave, res.search_bounds, velocity, trace, levels, counts,
                       group, gflags, flags, stats, 0)
    solver.close()
    assert stats["continuity_suspected"] == len(picks)
    assert stats["continuity_repaired"] == len(picks) and stats["continuity_unresolved"] == 0
    for b, f in picks:
        assert flags[b, f] & 3 == 3  # REVIEWED | REPAIRED
    # repaired traces equal the unplanted solve (review tolerance 1e-6)
    sel = tuple(np.array(picks).T)
    orig = res.phase_velocity[sel[0], :, sel[1]]
    got = velocity[sel[0], :, sel[1]]
    np.testing.assert_array_equal(np.isfinite(got), np.isfinite(orig))
    m = np.isfinite(orig)
    assert (np.abs(got[m] - orig[m]) / orig[m]).max() <= 2e-5
    # group velocities from _review_groups at the re-solved roots
    g_new, g_old = group[sel[0], :, sel[1]], res.group_velocity[sel[0], :, sel[1]]
    gm = np.isfinite(g_old) & np.isfinite(g_new)
    assert gm.sum() >= len(picks)
    assert (np.abs(g_new[gm] - g_old[gm]) / g_old[gm]).max() <= 1e-3
