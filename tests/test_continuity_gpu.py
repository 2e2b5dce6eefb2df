"""FP64 continuity recheck of the FP32-scan engine.

The screen (a trace is suspect when a mode with roots at both neighbouring
periods, within a log step of 0.25, is missing or leaves their +-5 % envelope --
the rule of cpp/cpu/continuity_screen.hpp:8-67) is restated here in numpy and
applied to the FP32-scan results without the recheck: the engine must re-scan
exactly those traces, return for them what the FP64 engine returns, and leave
every other trace untouched.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def screen(periods, velocity, flags):
    """Suspect traces [B, T] of a uniform batch (numpy restatement of the rule)."""
    B, K, T = velocity.shape
    order = np.argsort(periods, kind="stable")
    suspect = np.zeros((B, T), dtype=bool)
    for j in range(1, T - 1):
        f, l, r = order[j], order[j - 1], order[j + 1]
        if periods[l] == periods[f] or periods[r] == periods[f] or np.log(periods[r] / periods[l]) > .25:
            continue
        cl, cr, c = velocity[:, :, l], velocity[:, :, r], velocity[:, :, f]
        both = np.isfinite(cl) & np.isfinite(cr)
        bad = both & (~np.isfinite(c) | (c < .95 * np.fmin(cl, cr)) | (c > 1.05 * np.fmax(cl, cr)))
        suspect[:, f] = bad.any(axis=1)
    skip = (flags & (32768 | 4)) != 0  # already FP64-repaired, or unconverged
    return suspect & ~skip


@pytest.mark.parametrize("wave", [0, 1])
def test_continuity_recheck_rescans_exactly_the_suspects(wave):
    from modisp_b200 import _native, workloads
    batch = workloads.crustal_batch(256, workloads.SEED + 31, lvz_fraction=0.5)
    periods = np.geomspace(0.5, 50., 60)
    B, L = batch["thickness"].shape
    args = (batch["thickness"], batch["vp"], batch["vs"], batch["rho"], periods, None, 1e-10, 1., wave)
    out = {}
    for name, single, check in (("plain", 1, 0), ("checked", 1, 1), ("fp64", 0, 0)):
        o = _native.default_options()
        o.single_precision, o.group_velocity, o.continuity_check = single, 1, check
        eng = _native.Engine(0, B, L, periods.size, 5, o)
        try:
            out[name] = eng.run(*args, group=True)
        finally:
            eng.close()
    plain, checked, fp64 = out["plain"], out["checked"], out["fp64"]
    sus = screen(periods, plain["velocity"], plain["flags"])
    assert checked["stats"]["continuity_rescans"] == int(sus.sum())
    v0, v1, v64 = (x["velocity"].view(np.uint64) for x in (plain, checked, fp64))
    for b, f in zip(*np.nonzero(sus)):
        np.testing.assert_array_equal(v1[b, :, f], v64[b, :, f])
        assert checked["counts"][b, f] == fp64["counts"][b, f]
        assert checked["flags"][b, f] & 32768
        assert checked["levels"][b, f] == 22
    keep = ~sus
    np.testing.assert_array_equal(v1.transpose(0, 2, 1)[keep], v0.transpose(0, 2, 1)[keep])
    np.testing.assert_array_equal(checked["counts"][keep], plain["counts"][keep])
    g1, g64 = checked["group_velocity"].view(np.uint64), fp64["group_velocity"].view(np.uint64)
    for b, f in zip(*np.nonzero(sus)):
        np.testing.assert_array_equal(g1[b, :, f], g64[b, :, f])
    assert checked["stats"]["roots"] == int(np.isfinite(checked["velocity"]).sum())
