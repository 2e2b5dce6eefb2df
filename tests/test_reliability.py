"""Cross-period mode-reliability checks: the oracle pinned to the reference's own
outputs, the host-side argument checks and period plan (CPU), and the device
kernel against the oracle (GPU, bit-exact)."""
import glob
from pathlib import Path

import numpy as np
import pytest

import oracle.reliability as orel
from modisp_b200 import _native
from modisp_b200.reliability import ModeReliabilityFlag as F, check_mode_reliability, period_plan

GOLDEN = Path(__file__).resolve().parent / "golden"
OPTIONS = ("close_root_rtol", "max_relative_step", "prediction_rtol", "max_log_period_gap")
CASES = sorted(Path(p).stem.replace("reliability_", "") for p in glob.glob(str(GOLDEN / "reliability_*.npz")))


def load(case):
    f = np.load(GOLDEN / f"reliability_{case}.npz")
    inputs = dict(velocity=f["velocity"], periods=f["periods"],
                  trace_flags=f["trace_flags"] if "trace_flags" in f.files else None,
                  root_count=f["root_count"] if "root_count" in f.files else None,
                  **dict(zip(OPTIONS, f["options"].tolist())))
    expected = (f["flags"], f["assessed"], f["previous_index"], f["sorted_order"])
    return inputs, expected


def test_fixture_set_is_complete():
    assert len(CASES) >= 10 and "synthetic_full" in CASES and "lvz48_rayleigh" in CASES


@pytest.mark.parametrize("case", CASES)
def test_oracle_matches_reference_outputs(case):
    inputs, (flags, assessed, previous, order) = load(case)
    got = orel.check(inputs["velocity"], inputs["periods"], inputs["trace_flags"], inputs["root_count"],
                     *(inputs[k] for k in OPTIONS))
    np.testing.assert_array_equal(got[0], flags)
    np.testing.assert_array_equal(got[1], assessed)
    np.testing.assert_array_equal(got[2], previous)
    np.testing.assert_array_equal(got[3], order)


@pytest.mark.parametrize("case", CASES)
def test_period_plan_previous_and_order(case):
    inputs, (_, _, previous, order) = load(case)
    plan, plan_order, prev = period_plan(inputs["periods"], inputs["max_log_period_gap"])
    np.testing.assert_array_equal(prev, previous)
    np.testing.assert_array_equal(plan_order, order)
    # every distinct period lists exactly the sorted positions of its duplicates
    p = inputs["periods"]
    for t in range(p.size):
        if plan["kind"][t] & _native.PLAN_DUPLICATE:
            assert p[plan["prev"][t]] == p[t]
        else:
            dups = plan_order[plan["dup_begin"][t]:plan["dup_end"][t]]
            assert np.all(p[dups] == p[t]) and np.all(plan["kind"][dups] & _native.PLAN_DUPLICATE)


@pytest.mark.parametrize("bad, message", [
    (dict(velocity=np.ones((1, 1, 2)) + 1j), "real"),
    (dict(velocity=np.ones((1, 2))), r"expected velocity \[B,K,T\]"),
    (dict(periods=[1., -1.]), r"expected velocity \[B,K,T\]"),
    (dict(periods=[1., np.nan]), r"expected velocity \[B,K,T\]"),
    (dict(periods=[1.]), r"expected velocity \[B,K,T\]"),
    (dict(velocity=np.array([[[1., np.inf]]])), "positive finite"),
    (dict(velocity=np.array([[[1., 0.]]])), "positive finite"),
    (dict(trace_flags=np.array([[1., 0.]])), "trace_flags must be nonnegative integer"),
    (dict(trace_flags=np.array([[-1, 0]])), "trace_flags must be nonnegative integer"),
    (dict(trace_flags=np.zeros((2, 2), np.uint32)), "trace_flags must be nonnegative integer"),
    (dict(root_count=np.zeros((1, 2))), r"root_count must be integer"),
    (dict(close_root_rtol=0.), "close_root_rtol must be finite and positive"),
    (dict(max_relative_step=np.nan), "max_relative_step must be finite and positive"),
    (dict(prediction_rtol=[.1]), "prediction_rtol must be finite and positive"),
    (dict(max_log_period_gap=-1.), "max_log_period_gap must be finite and positive"),
])
def test_argument_checks(bad, message):
    args = dict(velocity=np.ones((1, 1, 2)), periods=[1., 2.])
    args.update(bad)
    v, p = args.pop("velocity"), args.pop("periods")
    with pytest.raises(ValueError, match=message):
        check_mode_reliability(v, p, **args)


def test_result_supplies_its_own_periods():
    class Result:
        phase_velocity = np.ones((1, 1, 2))
        period = np.array([1., 2.])
        trace_flags = np.zeros((1, 2), np.uint32)
        root_count = np.ones((1, 2), np.int32)
        close_root_rtol = .005
    with pytest.raises(ValueError, match="supplied by the result"):
        check_mode_reliability(Result(), [1., 2.])


def test_c_plan_builder_agrees_with_numpy_plan():
    _native.lib()
    rng = np.random.default_rng(5)
    p = np.round(np.exp(rng.uniform(-1., 4., 200)), 3)  # rounded: duplicates appear
    p[:3] = [1e100, np.nextafter(1e100, np.inf), np.nextafter(np.nextafter(1e100, np.inf), np.inf)]
    for gap in (.25, .05, 2.):
        plan, order, _ = period_plan(p, gap)
        cplan, corder = _native.reliability_plan(p, gap)
        np.testing.assert_array_equal(order, corder)
        for field in ("prev", "older", "kind", "dup_begin", "dup_end"):
            np.testing.assert_array_equal(plan[field], cplan[field], err_msg=field)
        # the logarithms are libm's in C and numpy's here: ratios agree to rounding
        np.testing.assert_allclose(plan["ratio"], cplan["ratio"], rtol=1e-14)


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_kernel_matches_reference_outputs(case):
    inputs, (flags, assessed, previous, order) = load(case)
    r = check_mode_reliability(inputs["velocity"], inputs["periods"], trace_flags=inputs["trace_flags"],
                               root_count=inputs["root_count"], **{k: inputs[k] for k in OPTIONS})
    np.testing.assert_array_equal(r.flags, flags)
    np.testing.assert_array_equal(r.assessed, assessed)
    np.testing.assert_array_equal(r.previous_index, previous)
    np.testing.assert_array_equal(r.sorted_order, order)


@pytest.mark.gpu
def test_reference_test_cases():
    periods = np.array([1.2, 1., 1.1, 1.1, 4.])
    v = np.array([[[1.02, 1., 1.01, 1.01, 1.2], [2.02, 2., 2.01, 2.01, 2.2]]])
    before = v.copy()
    r = check_mode_reliability(v, periods)
    np.testing.assert_array_equal(v, before)
    assert r.previous_index.tolist() == [2, -1, 1, 2, 0]
    assert np.all(r.flags[:, :, 1] & F.UNASSESSED) and np.all(r.flags[:, :, 4] & F.PERIOD_GAP)
    assert not r.assessed[:, :, 4].any()
    assert r.passes_checks[:, :, 0].all() and r.passes_checks[:, :, 3].all()
    v2 = np.array([[[1., 1.3, 1.8], [1.4, 1.8, np.nan], [2., 2.05, 2.1]]])
    r2 = check_mode_reliability(v2, [1., 1.1, 1.2], trace_flags=np.array([[0, 4096, 4]], dtype=np.uint32))
    assert np.any(r2.flags[:, :, 1] & F.RANK_AMBIGUOUS) and np.any(r2.flags[:, :, 1] & F.STEP_JUMP)
    assert np.all(r2.flags[:, :, 2] & F.ROOT_COUNT_CHANGE) and np.all(r2.flags[:, :, 2] & F.NUMERICAL_FAILURE)
    assert np.all(r2.flags[:, :, 1] & F.SEARCH_UNCERTAIN) and not r2.assessed[:, :, 2].any()
    s = r.summary()
    assert s["cells"] == 10 and s["flags"]["PERIOD_GAP"] == 2


@pytest.mark.gpu
def test_kernel_matches_oracle_on_random_batches():
    from tests.golden.make_golden import synthetic_reliability
    # K up to 12 takes a register-staged kernel for its exact K, larger K the general one
    for seed, (B, K, T) in enumerate(((64, 8, 31), (5, 1, 40), (3, 12, 7), (200, 3, 2), (6, 20, 9), (9, 13, 12))):
        v, p, tf, counts = synthetic_reliability(1000 + seed, B, K, T, duplicates=T > 4, gaps=T > 4)
        for opts in ({}, dict(close_root_rtol=.05, max_relative_step=.02, prediction_rtol=.002,
                              max_log_period_gap=.1)):
            for tfx, cx in ((tf, counts), (None, None)):
                r = check_mode_reliability(v, p, trace_flags=tfx, root_count=cx, **opts)
                full = dict(dict(zip(OPTIONS, (.005, .1, .05, .25))), **opts)
                want = orel.check(v, p, tfx, cx, *(full[k] for k in OPTIONS))
                np.testing.assert_array_equal(r.flags, want[0])
                np.testing.assert_array_equal(r.assessed, want[1])


@pytest.mark.gpu
def test_engine_results_and_device_entry_point():
    """The checks on a solved batch through DispersionBatch.check_modes, and the
    device-pointer entry point on the same arrays (bit-identical)."""
    import torch
    from modisp_b200 import Solver, workloads
    batch, periods, nmodes = workloads.config2(96)
    periods = np.concatenate([periods, periods[5:8]])  # duplicates: solved again, compared
    with Solver(precision="float32") as s:
        res = s(**batch, periods=periods, nmodes=nmodes, wave="rayleigh")
    r = res.check_modes()
    want = orel.check(res.phase_velocity, res.period, res.trace_flags, res.root_count, res.close_root_rtol)
    np.testing.assert_array_equal(r.flags, want[0])
    np.testing.assert_array_equal(r.assessed, want[1])
    B, K, T = res.phase_velocity.shape
    dev = torch.device("cuda", 0)
    v = torch.tensor(np.ascontiguousarray(res.phase_velocity, dtype=np.float64), device=dev)
    tf = torch.tensor(res.trace_flags.astype(np.int32), device=dev)
    cnt = torch.tensor(res.root_count.astype(np.int64), device=dev)
    fl = torch.zeros((B, K, T), dtype=torch.int16, device=dev)
    asd = torch.zeros((B, K, T), dtype=torch.uint8, device=dev)
    plan, order, _ = period_plan(res.period)
    stream = torch.cuda.current_stream().cuda_stream
    _native.mode_reliability_device(v.data_ptr(), tf.data_ptr(), cnt.data_ptr(), B, K, T, plan, order,
                                    res.close_root_rtol, .1, .05, fl.data_ptr(), asd.data_ptr(), stream)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(fl.cpu().numpy().view(np.uint16), want[0])
    np.testing.assert_array_equal(asd.cpu().numpy().astype(bool), want[1])
    # the same with the plan uploaded once (kernel only)
    plan_d = torch.tensor(plan.view(np.uint8), device=dev)
    order_d = torch.tensor(order, device=dev)
    fl.zero_()
    asd.zero_()
    _native.mode_reliability_planned(v.data_ptr(), tf.data_ptr(), cnt.data_ptr(), B, K, T, plan_d.data_ptr(),
                                     order_d.data_ptr(), res.close_root_rtol, .1, .05, fl.data_ptr(), asd.data_ptr(),
                                     stream)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(fl.cpu().numpy().view(np.uint16), want[0])
    np.testing.assert_array_equal(asd.cpu().numpy().astype(bool), want[1])


def test_c_entry_points_reject_bad_plans_before_any_device_work():
    """Every index the kernel follows is checked on the host first: a plan whose
    indices leave the period array, bad tolerances and bad periods are refused
    with a message (no GPU needed to see it)."""
    _native.lib()
    v = np.ones((1, 2, 3))
    plan, order, _ = period_plan(np.array([1., 2., 3.]))
    for field, value in (("prev", 7), ("older", -2), ("dup_end", 9)):
        bad = plan.copy()
        t = 2
        bad[field][t] = value
        if field == "older":
            bad["kind"][t] |= _native.PLAN_PREDICT
        with pytest.raises(RuntimeError, match="invalid period plan"):
            _native.mode_reliability(v, bad, order)
    bad_order = order.copy()
    bad_order[0] = 5
    with pytest.raises(RuntimeError, match="invalid period plan"):
        _native.mode_reliability(v, plan, bad_order)
    with pytest.raises(RuntimeError, match="tolerances must be finite and positive"):
        _native.mode_reliability(v, plan, order, close_root_rtol=-1.)
    with pytest.raises(RuntimeError, match="periods must be finite and positive"):
        _native.reliability_plan(np.array([1., np.nan]), .25)
