"""The continuity screen and the FP64 continuity recheck of the FP32-scan engine,
checked against the reference's own screen (``_cpu.continuity_screen``,
cpp/cpu/continuity_screen.hpp:8-67, from the reference CPU engine that the
oracle recipe builds).

* The screen's rules (ENVELOPE 16, CLOSE_FP32 32, PREDICTION 64, NO_BILATERAL 8)
  on synthetic results with defects planted on the host -- missing roots, roots
  outside the +-5 % envelope, adjacent modes within a few float32 ULPs, review
  predictions, unsorted and duplicate periods, period gaps on both sides of the
  0.25 log-step limit -- through md200_continuity_screen: flags identical to the
  reference's, bit for bit.
* The engine's own screen on its FP32-scan results: the flags it returns equal the
  reference screen's on the same results, its REVIEWED traces are exactly the
  reference's suspects, the re-scanned ones come back equal to the FP64 engine's,
  and every other trace is untouched.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SCREEN_BITS = 8 | 16 | 32 | 64


def synthetic_result(seed, B=64, K=6, T=30, unsorted=False, duplicates=False):
    rng = np.random.default_rng(seed)
    periods = np.geomspace(0.5, 10., T)  # two-period log steps of 0.21: every inner period bilateral
    if duplicates:
        periods[rng.choice(T - 1, 4, replace=False)] = periods[rng.choice(T - 1, 4, replace=False)]
    if unsorted:
        periods = rng.permutation(periods)
    base = rng.uniform(1., 2., (B, 1, 1)) * (1. + 0.4 * np.arange(K)[None, :, None]) \
        * (1. + 0.05 * np.log(periods)[None, None, :])
    v = base * rng.uniform(0.995, 1.005, (B, K, T))
    v[rng.random((B, K, T)) < 0.04] = np.nan                      # missing roots
    jump = rng.random((B, K, T)) < 0.03
    v[jump] *= rng.choice([0.9, 1.1], jump.sum())                  # envelope breaks
    b, t = rng.integers(0, B, 40), rng.integers(0, T, 40)
    k = rng.integers(1, K, 40)
    ulps = rng.integers(0, 40, 40)                                  # adjacent modes a few ULPs apart
    v32 = v.astype(np.float32)
    for bi, ki, ti, u in zip(b, k, t, ulps):
        x = np.float32(v32[bi, ki - 1, ti])
        if np.isfinite(x):
            v32[bi, ki, ti] = (x.view(np.uint32) + np.uint32(u)).view(np.float32)
    pred = np.where(rng.random((B, T)) < 0.05, 4096, 0).astype(np.uint32) | \
        np.where(rng.random((B, T)) < 0.2, 8, 0).astype(np.uint32)
    return periods, v32, pred


@pytest.mark.parametrize("case", ["sorted", "unsorted", "duplicates", "coarse"])
@pytest.mark.parametrize("precision", ["float32", "float64"])
@pytest.mark.parametrize("bilateral", [True, False])
def test_screen_rules_match_the_reference_screen(case, precision, bilateral, reference_engine):
    from modisp_b200 import _native
    periods, v32, pred = synthetic_result(11, unsorted=case == "unsorted", duplicates=case == "duplicates")
    if case == "coarse":  # two-period log steps on both sides of the 0.25 limit
        periods = 0.5 * np.exp(np.cumsum(np.random.default_rng(12).uniform(0.1, 0.15, periods.size)))
    v = v32 if precision == "float32" else v32.astype(np.float64) * (1 + 1e-12)
    for p in (None, pred):
        want, want_sus = reference_engine.continuity_screen(periods, v, p, bilateral)
        got, sus = _native.continuity_screen(periods, v, p, bilateral)
        np.testing.assert_array_equal(got, want)
        assert sus == want_sus
        assert np.any(got & 16) or not bilateral
        if precision == "float32" and bilateral:
            assert np.any(got & 32)


@pytest.mark.parametrize("wave", [0, 1])
def test_engine_screen_flags_and_rescans_match_the_reference_screen(wave, reference_engine):
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
            out[name] = eng.run(*args, group=True, continuity=True)
        finally:
            eng.close()
    plain, checked, fp64 = out["plain"], out["checked"], out["fp64"]
    assert not plain["continuity_flags"].any() and not fp64["continuity_flags"].any()  # unscreened engines
    want, _ = reference_engine.continuity_screen(periods, plain["velocity"].astype(np.float32), None, True)
    cf = checked["continuity_flags"]
    np.testing.assert_array_equal(cf & SCREEN_BITS, want)
    sus = (want & (16 | 32 | 64)) != 0
    np.testing.assert_array_equal((cf & 1) != 0, sus)  # REVIEWED
    rescan = sus & ((plain["flags"] & 32768) == 0)      # not already re-solved in FP64
    assert checked["stats"]["continuity_rescans"] == int(rescan.sum())
    v0, v1, v64 = (x["velocity"].view(np.uint64) for x in (plain, checked, fp64))
    g1, g64 = checked["group_velocity"].view(np.uint64), fp64["group_velocity"].view(np.uint64)
    for b, f in zip(*np.nonzero(rescan)):
        np.testing.assert_array_equal(v1[b, :, f], v64[b, :, f])
        np.testing.assert_array_equal(g1[b, :, f], g64[b, :, f])
        assert checked["counts"][b, f] == fp64["counts"][b, f]
        assert checked["flags"][b, f] & 32768 and checked["levels"][b, f] == 22
        changed = plain["counts"][b, f] != fp64["counts"][b, f] or not np.allclose(
            plain["velocity"][b, :, f], fp64["velocity"][b, :, f], rtol=1e-10, atol=0, equal_nan=True)
        assert bool(cf[b, f] & 2) == changed  # REPAIRED
    keep = ~rescan
    np.testing.assert_array_equal(v1.transpose(0, 2, 1)[keep], v0.transpose(0, 2, 1)[keep])
    np.testing.assert_array_equal(checked["counts"][keep], plain["counts"][keep])
    assert checked["stats"]["roots"] == int(np.isfinite(checked["velocity"]).sum())


def test_public_api_returns_continuity_flags():
    import modisp_b200 as md
    from modisp_b200 import workloads
    batch = workloads.crustal_batch(32, workloads.SEED + 32)
    periods = np.geomspace(0.5, 50., 40)
    r = md.dispersion_batch(batch["thickness"], batch["vp"], batch["vs"], batch["rho"], periods, 5,
                            precision="float32", accuracy="high")
    assert r.continuity_flags is not None and r.continuity_flags.shape == (32, 40)
    assert r.continuity_flags.dtype == np.uint8
    r64 = md.dispersion_batch(batch["thickness"], batch["vp"], batch["vs"], batch["rho"], periods, 5)
    assert r64.continuity_flags is None
