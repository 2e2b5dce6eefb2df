"""Pin the oracle (CPU, no GPU needed).

The C restatement (oracle/md_oracle.c) must reproduce the reference CPU engine
bit for bit on secular values and search windows, agree with the reference's
frozen fixtures, and its complex-step group velocity must be the limit the
reference's finite-difference estimator converges to as its tolerance tightens.
"""
import numpy as np
import pytest

from conftest import GOLDEN, load_golden

RNG = np.random.default_rng(20261203)


def _random_model(rng, water=False, lvz=False):
    L = int(rng.integers(2, 14))
    vs = np.sort(rng.uniform(0.3, 4.5, L))
    vp = vs * rng.uniform(1.7, 2.0, L)
    rho = 1.74 * vp ** 0.25
    h = rng.uniform(0.1, 3.0, L)
    h[-1] = 0.
    if lvz and L > 3:
        vs[2] = vs[1] * 0.7
        vp[2] = vs[2] * 1.8
    if water:
        vs[0], vp[0], rho[0] = 0., 1.5, 1.02
    return h, vp, vs, rho


@pytest.mark.parametrize("trial", range(40))
def test_secular_values_bitwise_equal_to_reference(trial, oracle_lib, reference_engine):
    rng = np.random.default_rng(trial)
    water = trial % 5 == 0
    h, vp, vs, rho = _random_model(rng, water=water, lvz=trial % 3 == 0)
    wave = 0 if water else trial % 2
    period = float(rng.uniform(0.2, 40.))
    c = np.sort(rng.uniform(0.05, vs[-1], 48))
    c[:2] = [vs[1], vp[0]]  # exact body velocities hit the equality branches
    f_ref, g_ref = reference_engine.secular_shape(h, vp, vs, rho, period, c, wave, 0)
    f, g = oracle_lib.secular(h, vp, vs, rho, period, c, wave, shape=True)
    np.testing.assert_array_equal(f.view(np.uint64), f_ref.view(np.uint64))
    np.testing.assert_array_equal(g.view(np.uint64), g_ref.view(np.uint64))


@pytest.mark.parametrize("wave", [0, 1])
def test_bounds_bitwise_equal_to_reference(wave, oracle_lib, reference_engine):
    rng = np.random.default_rng(7 + wave)
    B, L = 40, 9
    vs = np.sort(rng.uniform(0.3, 4.5, (B, L)), axis=1)
    vp = vs * rng.uniform(1.7, 2.0, (B, L))
    rho = 1.74 * vp ** 0.25
    h = rng.uniform(0.2, 3., (B, L))
    h[:, -1] = 0.
    h[::7, 3] = 0.  # zero-thickness interior rows are skipped by the window rule
    if wave == 0:
        vs[::5, 0], vp[::5, 0], rho[::5, 0] = 0., 1.5, 1.02
    ref = reference_engine.bounds(h, vp, vs, rho, wave, None, None)
    mine = oracle_lib.bounds(h, vp, vs, rho, wave)
    np.testing.assert_array_equal(mine.view(np.uint64), ref.view(np.uint64))


def test_group_velocity_is_the_limit_of_the_reference_estimator(oracle_lib):
    """Reference FD group velocity converges to the complex-step value as group_rtol shrinks."""
    g = load_golden("ref_quickstart_rayleigh")
    h, vp, vs, rho = (g[k][0] for k in ("thickness", "vp", "vs", "rho"))
    lo, hi = g["search_bounds"][0]
    errors = []
    for f, period in enumerate(g["periods"]):
        v = g["phase_velocity"][0, :, f]
        roots = v[np.isfinite(v)]
        wl, wh, _ = oracle_lib.group_windows(roots, lo, hi)
        for m, c in enumerate(roots):
            if g["group_velocity_flags"][0, m, f]:
                continue
            u = oracle_lib.group(h, vp, vs, rho, period, c, wl[m], wh[m], 0)
            errors.append(abs(u - g["group_velocity"][0, m, f]) / u)
    # the reference's estimator at group_rtol = 1e-3 targets a relative error of 2.5e-4
    assert errors and max(errors) < 2.5e-4


def test_group_velocity_tightens_with_reference_tolerance(oracle_lib, reference_engine):
    model_h = np.array([0.3, 0.]); vp = np.array([2., 5.]); vs = np.array([.8, 2.8]); rho = np.array([2., 2.6])
    periods = np.geomspace(0.1, 10., 30)
    worst = []
    for rtol in (1e-3, 1e-5, 1e-7):
        out = oracle_lib.reference_solve(model_h, vp, vs, rho, periods, 2, wave=0, tol=1e-12,
                                         group_velocity=True, group_rtol=rtol)
        lo, hi = out["search_bounds"][0]
        err = 0.
        for f, period in enumerate(periods):
            v = out["phase_velocity"][0, :, f]
            roots = v[np.isfinite(v)]
            wl, wh, _ = oracle_lib.group_windows(roots, lo, hi)
            for m, c in enumerate(roots):
                if out["group_velocity_flags"][0, m, f] == 0:
                    u = oracle_lib.group(model_h, vp, vs, rho, period, c, wl[m], wh[m], 0)
                    err = max(err, abs(u - out["group_velocity"][0, m, f]) / u)
        worst.append(err)
    assert worst[0] > worst[1] > worst[2]
    assert worst[2] < 1e-10


def test_half_space_rayleigh_speed_and_group(oracle_lib):
    """Homogeneous half-space: one root at the Rayleigh speed, U = c (no dispersion)."""
    h = np.array([1.0, 0.]); vp = np.array([6., 6.]); vs = np.array([3.5, 3.5]); rho = np.array([2.7, 2.7])
    lo, hi = oracle_lib.bounds(h, vp, vs, rho, 0)[0]
    n, roots = oracle_lib.dense_roots(h, vp, vs, rho, 1.0, lo, hi, 3)
    assert n == 1
    # Rayleigh speed of Poisson-like vp/vs: bisection of the Rayleigh cubic
    ratio = (3.5 / 6.) ** 2
    x = np.roots([1., -8., 24. - 16. * ratio, -16. * (1. - ratio)])
    x = np.real(x[(np.abs(np.imag(x)) < 1e-12) & (np.real(x) > 0) & (np.real(x) < 1)])[0]
    assert abs(roots[0] - 3.5 * np.sqrt(x)) < 1e-9
    u = oracle_lib.group(h, vp, vs, rho, 1.0, roots[0], lo, hi, 0)
    assert abs(u - roots[0]) / roots[0] < 1e-10


def test_dense_search_matches_reference_roots(oracle_lib):
    """The dense-grid restatement recovers the reference's root sets on the quickstart model."""
    for wave, name in ((0, "ref_quickstart_rayleigh"), (1, "ref_quickstart_love")):
        g = load_golden(name)
        h, vp, vs, rho = (g[k][0] for k in ("thickness", "vp", "vs", "rho"))
        lo, hi = g["search_bounds"][0]
        K = int(g["nmodes"]) + 2
        for f, period in enumerate(g["periods"]):
            n, roots = oracle_lib.dense_roots(h, vp, vs, rho, period, lo, hi, K, 1e-12, wave)
            assert n == g["root_count"][0, f]
            ref = g["phase_velocity"][0, :, f]
            np.testing.assert_allclose(roots[:ref.size][np.isfinite(ref)], ref[np.isfinite(ref)], rtol=1e-11)


@pytest.mark.parametrize("name", sorted(p.stem for p in GOLDEN.glob("fixture_0*.npz")))
def test_reference_fixture_roots_are_roots_of_the_oracle(name, oracle_lib):
    """Every frozen reference root is a sign change of the restated secular function."""
    g = load_golden(name)
    h, vp, vs, rho = (np.atleast_2d(g[k]) for k in ("thickness", "vp", "vs", "rho"))
    wave = 1 if str(g["wave"]) == "love" else 0
    v = g["phase_velocity"]
    checked = 0
    for b in range(v.shape[0]):
        for f, period in enumerate(g["periods"]):
            for c in v[b, :, f][np.isfinite(v[b, :, f])]:
                a, z = oracle_lib.secular(h[b], vp[b], vs[b], rho[b], period, [c * (1 - 1e-6), c * (1 + 1e-6)], wave)
                assert np.signbit(a) != np.signbit(z) or a == 0. or z == 0.
                checked += 1
    assert checked > 0


def test_reference_fixture_windows_match_oracle(oracle_lib):
    for path in sorted(GOLDEN.glob("fixture_0*.npz")):
        g = load_golden(path.stem)
        if np.isfinite(g["cmin"]) or np.isfinite(g["cmax"]):
            continue
        wave = 1 if str(g["wave"]) == "love" else 0
        mine = oracle_lib.bounds(np.atleast_2d(g["thickness"]), np.atleast_2d(g["vp"]),
                                 np.atleast_2d(g["vs"]), np.atleast_2d(g["rho"]), wave)
        np.testing.assert_array_equal(mine, g["search_bounds"])


def test_witness_roots_are_recovered_by_reference_engine(oracle_lib, reference_engine):
    """The independent witnesses (FP64 CPS/disba, pinned QEDispInv) of the reference
    suite, some with near-kissing pairs 4e-5 apart, pin the root-set oracle."""
    for path in sorted(GOLDEN.glob("fixture_witness_*.npz")):
        g = load_golden(path.stem)
        expected = g["reference_hi"].ravel()
        # at its default high tolerance (1e-6); at 1e-12 the reference's shape search
        # exhausts its depth on witness 9951 and its fallback ladder misses the pair
        out = oracle_lib.reference_solve(g["thickness"], g["vp"], g["vs"], g["rho"], g["periods"],
                                         expected.size, wave=0, tol=1e-6)
        np.testing.assert_allclose(out["phase_velocity"].ravel(), expected, rtol=2e-6)


def test_b10000_cropped_roots_are_recovered_by_reference_engine(oracle_lib, reference_engine):
    for path in sorted(GOLDEN.glob("fixture_B10000_*.npz")):
        g = load_golden(path.stem)
        expected = g["reference"].ravel()[:3]
        h, vp, vs, rho = (np.atleast_2d(g[k]) for k in ("thickness", "vp", "vs", "rho"))
        bnd = reference_engine.bounds(h, vp, vs, rho, 0, .2, None)
        solver = reference_engine.CpuSolver(4, 0, 0., .005, True, .001, 0, 1, 1)
        v = solver.run(h, vp, vs, rho, g["periods"], bnd, 3, 0, False, 1e-6, 1.)[0]
        np.testing.assert_allclose(v.ravel(), expected, rtol=2e-6)


def test_dense_restatement_misses_what_a_plain_grid_misses(oracle_lib):
    """A uniform grid coarser than a close pair's gap cannot see the pair: the reason
    the engine probes same-sign troughs (witness model 9384 has a 3.6e-5 pair)."""
    g = load_golden("fixture_witness_model9384_period11")
    h, vp, vs, rho = g["thickness"], g["vp"], g["vs"], g["rho"]
    lo, hi = oracle_lib.bounds(h, vp, vs, rho, 0)[0]
    expected = g["reference_hi"].ravel()
    n, roots = oracle_lib.dense_roots(h, vp, vs, rho, float(g["periods"][0]), lo, hi, expected.size)
    assert n == expected.size and not np.allclose(roots, expected, rtol=2e-6)


def test_complex_step_matches_finite_differences(oracle_lib):
    g = load_golden("ref_crustal48_rayleigh")
    b, f, m, j = 3, 30, 0, 1
    h, vp, vs, rho = (g[k][b] for k in ("thickness", "vp", "vs", "rho"))
    c = g["phase_velocity"][b, m, f]
    period = g["periods"][f]
    dth, dfdc = oracle_lib.parameter_derivatives(h, vp, vs, rho, period, c, 0)
    # central finite differences of F in vs of layer j (scale-free ratio test against dF/dc)
    eps = 1e-6 * vs[j]
    vp1, vs1 = vp.copy(), vs.copy()
    vs1[j] += eps
    fp = oracle_lib.secular(h, vp1, vs1, rho, period, [c], 0)[0]
    vs1[j] -= 2 * eps
    fm = oracle_lib.secular(h, vp1, vs1, rho, period, [c], 0)[0]
    cp = oracle_lib.secular(h, vp, vs, rho, period, [c * (1 + 1e-7)], 0)[0]
    cm = oracle_lib.secular(h, vp, vs, rho, period, [c * (1 - 1e-7)], 0)[0]
    ratio_fd = ((fp - fm) / (2 * eps)) / ((cp - cm) / (2e-7 * c))
    assert abs(ratio_fd) > 1e-3
    assert abs(ratio_fd - dth[2, j] / dfdc) < 1e-4 * abs(ratio_fd)


@pytest.mark.parametrize("wave", [0, 1])
def test_phase_jacobian_matches_reference_finite_differences(wave, oracle_lib, reference_engine):
    """The oracle's implicit-function Jacobian dc/dm = -F_m / F_c equals central
    differences (step 1e-6 relative) of the reference solver's roots."""
    rng = np.random.default_rng(41 + wave)
    n = 6
    vs = np.linspace(rng.uniform(.3, 1.), rng.uniform(3.5, 4.7), n + 1) * rng.uniform(.9, 1.1, n + 1)
    vs[-1] = max(vs[-1], vs[:-1].max() * 1.02)
    vp = vs * rng.uniform(1.7, 2., n + 1)
    rho = 1.74 * vp ** .25
    h = rng.uniform(.2, 3., n + 1)
    h[-1] = 0.
    periods = np.geomspace(1., 40., 6)
    roots, fd = oracle_lib.reference_fd_phase_jacobian(h, vp, vs, rho, periods, 3, wave)
    checked = 0
    for m in range(3):
        for f, period in enumerate(periods):
            c = roots[m, f]
            if not np.isfinite(c):
                continue
            jac = oracle_lib.phase_jacobian(h, vp, vs, rho, period, c, wave)
            scale = np.abs(jac).max()
            assert np.abs(jac - fd[m, f]).max() < 1e-6 * scale, (m, f)
            checked += 1
    assert checked >= 10


def test_group_jacobian_differences_are_converged(oracle_lib):
    """Central differences of the polished group velocity agree at two step sizes
    (1e-6 and 1e-5 relative) to well inside the tolerance the engine is held to."""
    h = np.array([0.3, 1.2, 0.]); vp = np.array([2., 3.5, 6.]); vs = np.array([.8, 2., 3.4])
    rho = 1.74 * vp ** .25
    for wave in (0, 1):
        lo, hi = oracle_lib.bounds(h, vp, vs, rho, wave)[0]
        n, roots = oracle_lib.dense_roots(h, vp, vs, rho, 3.0, lo, hi, 3, 1e-14, wave)
        for c in roots[:n]:
            a = oracle_lib.group_jacobian_fd(h, vp, vs, rho, 3.0, c, wave, rel=1e-6)
            b = oracle_lib.group_jacobian_fd(h, vp, vs, rho, 3.0, c, wave, rel=1e-5)
            assert np.abs(a - b).max() < 1e-7 * np.abs(a).max()


@pytest.mark.parametrize("name", ["jac_config4_rayleigh", "jac_config4_love", "jac_water_rayleigh"])
def test_jacobian_fixtures_agree_with_the_oracle(name, oracle_lib):
    """The committed finite-difference Jacobians of the reference solver agree with
    the oracle's implicit-function Jacobians at every recorded root."""
    g = load_golden(name)
    wave = int(g["wave"])
    v = g["phase_velocity"]
    worst, checked = 0., 0
    for b in range(v.shape[0]):
        model = [g[k][b] for k in ("thickness", "vp", "vs", "rho")]
        for m in range(v.shape[1]):
            for f, period in enumerate(g["periods"]):
                c = v[b, m, f]
                if not np.isfinite(c):
                    continue
                jac = oracle_lib.phase_jacobian(*model, period, c, wave)
                worst = max(worst, np.abs(jac - g["jac_phase_fd"][b, m, f]).max() / np.abs(jac).max())
                checked += 1
    assert checked > 50 and worst < 1e-6


@pytest.mark.parametrize("case", ["crustal12", "lvz12", "lowc6", "deep4"])
def test_uniform_stage2_restatement_is_the_reference(case, oracle_lib):
    """mdo_uniform_refine on the reference's own stage 1 values (the fixtures of
    tests/golden/make_uniform_golden.py, made by the reference's CUDA legacy path)
    returns its roots bit for bit, its trace flags and its six counters."""
    g = load_golden(f"uniform_{case}")
    model = [g[k] for k in ("thickness", "vp", "vs", "rho")]
    v, flags, stats = oracle_lib.uniform_refine(g["rows"], *model, g["periods"], int(g["nmodes"]), float(g["cmin"]),
                                                float(g["cmax"]), float(g["c_tol_rel"]), float(g["f_accept"]))
    ref = g["phase_velocity"]
    np.testing.assert_array_equal(np.isfinite(v), np.isfinite(ref))
    np.testing.assert_array_equal(v[np.isfinite(ref)], ref[np.isfinite(ref)])
    np.testing.assert_array_equal(flags, g["trace_flags"])
    assert stats == {str(k): int(x) for k, x in zip(g["stat_names"], g["stats"])}
