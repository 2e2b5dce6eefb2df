"""Ragged batches (per-model periods and mode counts in one set of launches).

* a ragged batch whose models all share one period set and mode count returns
  exactly (bit for bit) what the uniform engine returns;
* a mixed ragged batch returns exactly what solving each model alone, with its
  own periods and modes, returns;
* config-5-shaped models (30-100 thin layers, own period windows, 1-10 modes)
  match the reference engine run per model: masks and counts identical, phase
  velocities within 1e-9;
* the device-pointer entry point matches the host one.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _engine(B, L, T, nm, single=True):
    from modisp_b200 import _native
    o = _native.default_options()
    o.single_precision = int(single)
    o.group_velocity = 1
    return _native.Engine(0, B, L, T, nm, o)


@pytest.mark.parametrize("wave", [0, 1])
def test_uniform_ragged_batch_equals_uniform_run(wave):
    from modisp_b200 import workloads
    batch = workloads.crustal_batch(96, workloads.SEED + 11)
    periods = np.geomspace(0.5, 50., 40)
    B, L = batch["thickness"].shape
    eng = _engine(B, L, periods.size, 5)
    try:
        uni = eng.run(batch["thickness"], batch["vp"], batch["vs"], batch["rho"], periods, None, 1e-10, 1., wave,
                      group=True)
        off = np.arange(B + 1, dtype=np.int32) * periods.size
        rag = eng.run_ragged(batch["thickness"], batch["vp"], batch["vs"], batch["rho"], off, np.tile(periods, B),
                             np.full(B, 5, np.int32), 1e-10, 1., wave, group=True)
    finally:
        eng.close()
    np.testing.assert_array_equal(rag["velocity"].reshape(B, 5, -1).view(np.uint64), uni["velocity"].view(np.uint64))
    np.testing.assert_array_equal(rag["group_velocity"].reshape(B, 5, -1).view(np.uint64),
                                  uni["group_velocity"].view(np.uint64))
    np.testing.assert_array_equal(rag["flags"].reshape(B, -1), uni["flags"])
    np.testing.assert_array_equal(rag["counts"].reshape(B, -1), uni["counts"])
    np.testing.assert_array_equal(rag["levels"].reshape(B, -1), uni["levels"])


@pytest.mark.parametrize("single", [True, False])
def test_mixed_ragged_batch_equals_per_model_runs(single):
    from modisp_b200 import workloads
    from modisp_b200.ragged import dispersion_ragged
    batch = workloads.crustal_batch(24, workloads.SEED + 12)
    rng = np.random.default_rng(5)
    periods = [np.geomspace(rng.uniform(0.3, 3.), rng.uniform(5., 60.), int(rng.integers(1, 30))) for _ in range(24)]
    modes = rng.integers(1, 8, 24)
    res = dispersion_ragged(batch["thickness"], batch["vp"], batch["vs"], batch["rho"], periods, modes,
                            precision="mixed" if single else "float64")
    L = batch["thickness"].shape[1]
    for b in range(24):
        eng = _engine(1, L, periods[b].size, int(modes[b]), single)
        try:
            one = eng.run(batch["thickness"][b:b + 1], batch["vp"][b:b + 1], batch["vs"][b:b + 1],
                          batch["rho"][b:b + 1], periods[b], None, 1e-10, 1., 0, group=True)
        finally:
            eng.close()
        np.testing.assert_array_equal(res.phase_velocity_of(b).view(np.uint64), one["velocity"][0].view(np.uint64))
        np.testing.assert_array_equal(res.group_velocity_of(b).view(np.uint64),
                                      one["group_velocity"][0].view(np.uint64))
        np.testing.assert_array_equal(res.root_count_of(b), one["counts"][0])
        np.testing.assert_array_equal(res.trace_flags_of(b), one["flags"][0])


CONFIG5_SAMPLE = 256


@pytest.mark.parametrize("wave", [0, 1])
def test_config5_sample_matches_reference(wave):
    """256 models of the large uneven workload (30-100 thin layers, own 50-120
    periods in 0.2-100 s, 1-10 modes) per wave, one ragged batch in each engine
    (FP32 scan and plain FP64), against the reference CPU engine run live per
    model on all host cores: masks and counts identical, phase within 1e-9."""
    import oracle
    from modisp_b200 import workloads
    from modisp_b200.ragged import dispersion_ragged
    if oracle.reference() is None:
        pytest.skip("reference CPU engine not built")
    batch, periods, modes = workloads.gradient_batch(CONFIG5_SAMPLE, seed=workloads.SEED + 5 + wave)
    res = {p: dispersion_ragged(batch["thickness"], batch["vp"], batch["vs"], batch["rho"], periods, modes,
                                wave="love" if wave else "rayleigh", precision=p) for p in ("mixed", "float64")}
    threads = len(os.sched_getaffinity(0))
    for b in range(CONFIG5_SAMPLE):
        sl = slice(b, b + 1)
        ref = oracle.reference_solve(batch["thickness"][sl], batch["vp"][sl], batch["vs"][sl], batch["rho"][sl],
                                     periods[b], int(modes[b]), wave=wave, tol=1e-10, threads=threads)
        rv = ref["phase_velocity"][0]
        m = np.isfinite(rv)
        for p, r in res.items():
            v = r.phase_velocity_of(b)
            np.testing.assert_array_equal(np.isfinite(v), m, err_msg=f"model {b} {p}")
            np.testing.assert_array_equal(r.root_count_of(b), ref["root_count"][0], err_msg=f"model {b} {p}")
            assert np.all(np.abs(v[m] - rv[m]) <= 1e-9 * rv[m]), f"model {b} {p}"


def test_row_periods_through_the_plugin():
    """One period per model ([B, 1] periods, SUPPORTS_ROW_PERIODS) equals solving
    each model at its period in a uniform batch, windows included."""
    from modisp_b200 import plugin, workloads
    batch = workloads.crustal_batch(40, workloads.SEED + 13)
    B, L = batch["thickness"].shape
    rng = np.random.default_rng(8)
    per = rng.uniform(0.5, 40., (B, 1))
    bounds = np.zeros((B, 2))
    bounds[:, 1] = np.inf
    bounds[::3, 1] = 3.0  # some truncated windows
    s = plugin.QeSolver(B, L, 1, 4, 0, 0., .005, True, .001, 0, 1, 1, False, True, .001, False, 4)
    try:
        v, flags, _, levels, counts, extras = s.run(batch["thickness"], batch["vp"], batch["vs"], batch["rho"], per,
                                                    bounds, 1e-10, 1., 0)
    finally:
        s.close()
    assert v.shape == (B, 4, 1) and counts.shape == (B, 1)
    for b in range(B):
        one = plugin.QeSolver(1, L, 1, 4, 0, 0., .005, True, .001, 0, 1, 1, False, True, .001, False, 4)
        try:
            v1, f1, _, l1, c1, e1 = one.run(batch["thickness"][b:b + 1], batch["vp"][b:b + 1], batch["vs"][b:b + 1],
                                            batch["rho"][b:b + 1], per[b], bounds[b:b + 1], 1e-10, 1., 0)
        finally:
            one.close()
        np.testing.assert_array_equal(v[b].view(np.uint64), v1[0].view(np.uint64))
        np.testing.assert_array_equal(extras["group_velocity"][b].view(np.uint64),
                                      e1["group_velocity"][0].view(np.uint64))
        assert counts[b, 0] == c1[0, 0] and flags[b, 0] == f1[0, 0]


def test_ragged_device_entry_matches_host():
    import torch
    from modisp_b200 import workloads
    batch, periods, modes = workloads.gradient_batch(12, seed=workloads.SEED + 9)
    B, L = batch["thickness"].shape
    off = np.zeros(B + 1, np.int32)
    off[1:] = np.cumsum([p.size for p in periods])
    flat = np.concatenate(periods)
    md = np.asarray(modes, np.int32)
    cells = md.astype(np.int64) * np.diff(off)
    outb = np.zeros(B, np.int64)
    outb[1:] = np.cumsum(cells)[:-1]
    T_max, nm = int(np.diff(off).max()), int(md.max())
    eng = _engine(B, L, T_max, nm)
    try:
        host = eng.run_ragged(batch["thickness"], batch["vp"], batch["vs"], batch["rho"], off, flat, md, 1e-10, 1.,
                              0, group=True)
        dev = torch.device("cuda", 0)
        t = {k: torch.tensor(v, device=dev) for k, v in
             dict(h=batch["thickness"], vp=batch["vp"], vs=batch["vs"], rho=batch["rho"], off=off, per=flat, md=md,
                  outb=outb).items()}
        n = int(cells.sum())
        vel = torch.empty(n, dtype=torch.float64, device=dev)
        grp = torch.empty_like(vel)
        gfl = torch.empty(n, dtype=torch.int32, device=dev)
        fl, lv, ct = (torch.empty(flat.size, dtype=torch.int32, device=dev) for _ in range(3))
        stream = torch.cuda.current_stream().cuda_stream
        eng.run_ragged_device(t["h"].data_ptr(), t["vp"].data_ptr(), t["vs"].data_ptr(), t["rho"].data_ptr(), B,
                              flat.size, t["off"].data_ptr(), t["per"].data_ptr(), t["md"].data_ptr(),
                              t["outb"].data_ptr(), 1e-10, 1., 0, vel.data_ptr(), fl.data_ptr(), lv.data_ptr(),
                              ct.data_ptr(), grp.data_ptr(), gfl.data_ptr(), stream=stream)
        torch.cuda.synchronize()
    finally:
        eng.close()
    np.testing.assert_array_equal(vel.cpu().numpy().view(np.uint64), host["velocity"].view(np.uint64))
    np.testing.assert_array_equal(grp.cpu().numpy().view(np.uint64), host["group_velocity"].view(np.uint64))
    np.testing.assert_array_equal(ct.cpu().numpy(), host["counts"])
