"""Anchor continuation (frequency_strategy="anchor_continuation"; the reference's
cpp/common/continuation.hpp:12-212, cpp/cpu/solver.cpp:603-705).

Anchors are solved by the full search; the periods between them are predicted
from the anchors' roots and slopes, refined locally and audited, and any doubtful
one falls back to the full FP64 search.  The results must be the full search's:
mode masks and root counts identical, phase velocities within 1e-9, on a
dense-period crustal / low-velocity-layer batch (uniform) and on a sample of the
large uneven workload (ragged, every model over its own periods).  Prediction
flags follow the reference's PredictionFlag: anchors ANCHOR, targets ACCEPTED or
FALLBACK with the reason bits.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-10


def compare(a_vel, a_counts, b_vel, b_counts, where):
    np.testing.assert_array_equal(np.isfinite(a_vel), np.isfinite(b_vel), err_msg=f"{where}: masks")
    np.testing.assert_array_equal(a_counts, b_counts, err_msg=f"{where}: counts")
    m = np.isfinite(b_vel)
    rel = np.abs(a_vel[m] - b_vel[m]) / b_vel[m]
    assert rel.max(initial=0.) <= 1e-9, f"{where}: max |dc|/c {rel.max():.3e}"


@pytest.mark.parametrize("precision", ["float64", "mixed"])
@pytest.mark.parametrize("wave", ["rayleigh", "love"])
def test_continuation_equals_the_full_search(wave, precision):
    import modisp_b200 as md
    from modisp_b200 import workloads
    batch = workloads.crustal_batch(96, workloads.SEED + 61, lvz_fraction=0.3)
    periods = np.geomspace(0.5, 50., 120)
    args = (batch["thickness"], batch["vp"], batch["vs"], batch["rho"], periods, 5, wave)
    opts = dict(accuracy="balanced", c_tol_rel=TOL, group_velocity=True, precision=precision)
    full = md.dispersion_batch(*args, **opts)
    with md.Solver(frequency_strategy="anchor_continuation", **opts) as s:
        cont = s(*args)
        stats = s.stats()
    assert cont.frequency_strategy_used == "anchor_continuation"
    compare(cont.phase_velocity, cont.root_count, full.phase_velocity, full.root_count, f"{wave} {precision}")
    pf = cont.prediction_flags
    anchors = (pf & 1) != 0
    accepted = (pf & 2) != 0
    fallback = (pf & 4) != 0
    assert np.all(anchors ^ accepted ^ fallback)  # every trace exactly one of them
    assert np.all(anchors[:, 0]) and np.all(anchors[:, -1])
    assert stats["continuation_accepted"] == int(accepted.sum())
    assert stats["continuation_fallbacks"] == int(fallback.sum())
    # the predictions do serve: the reference's own continuation accepts 27 %
    # (Rayleigh) and 17 % (Love) of these targets (CPU engine, same batch)
    assert accepted.sum() > 0.1 * (accepted.sum() + fallback.sum())
    np.testing.assert_array_equal((cont.trace_flags[accepted] & 65536) != 0, True)  # CONTINUATION_APPROXIMATE
    np.testing.assert_array_equal(cont.search_level[accepted], 23)
    # group velocity of the accepted roots: the same analytic derivative at nearly the same roots
    g = np.isfinite(cont.group_velocity) & np.isfinite(full.group_velocity)
    np.testing.assert_array_equal(np.isfinite(cont.group_velocity), np.isfinite(full.group_velocity))
    assert np.max(np.abs(cont.group_velocity[g] - full.group_velocity[g]) / full.group_velocity[g]) <= 1e-8


def test_high_accuracy_keeps_the_independent_search():
    import modisp_b200 as md
    from modisp_b200 import workloads
    batch = workloads.crustal_batch(8, workloads.SEED + 62)
    with md.Solver(frequency_strategy="anchor_continuation", accuracy="high") as s:
        r = s(batch["thickness"], batch["vp"], batch["vs"], batch["rho"], np.geomspace(1., 20., 30), 3)
    assert r.frequency_strategy_used == "independent"
    assert r.frequency_strategy_reason == "high accuracy retains independent search"
    np.testing.assert_array_equal(r.prediction_flags, 8)  # BYPASSED


@pytest.mark.parametrize("wave", ["rayleigh", "love"])
def test_continuation_on_the_large_uneven_workload(wave):
    from modisp_b200 import workloads
    from modisp_b200.ragged import dispersion_ragged
    batch, periods, modes = workloads.gradient_batch(128, seed=workloads.SEED + 70)
    args = (batch["thickness"], batch["vp"], batch["vs"], batch["rho"], periods, modes, wave)
    full = dispersion_ragged(*args)
    cont = dispersion_ragged(*args, frequency_strategy="anchor_continuation")
    compare(cont.phase_velocity, cont.root_count, full.phase_velocity, full.root_count, f"config5 {wave}")
    st = cont.stats
    assert st["continuation_accepted"] > 0
    assert st["continuation_anchors"] + st["continuation_accepted"] + st["continuation_fallbacks"] == \
        sum(p.size for p in periods)
