"""Phase- and group-velocity Jacobians on the GPU (adjoint kernel, C ABI and autograd).

Checked against three oracles:
  * the reference solver's own roots differentiated by central differences
    (committed fixtures, step 1e-6 relative; FD noise ~1e-8 of the row scale);
  * the oracle's implicit-function Jacobian from long-double complex-step
    derivatives of the secular function (tight: 1e-9 of the row scale);
  * central differences of the oracle's polished group velocity for dU/dm
    (1e-6 of the row scale; the differences themselves converge to ~1e-10).
Errors are measured per root as max |J - J_ref| / max |J_ref| over its 4 x L row.
"""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

PHASE_TOL_ORACLE = 1e-9
PHASE_TOL_FD = 1e-6
GROUP_TOL_FD = 1e-6


def _engine(B, L, T, nm, single=False):
    from modisp_b200 import _native
    o = _native.default_options()
    o.single_precision = int(single)
    o.group_velocity = 1
    return _native.Engine(0, B, L, T, nm, o)


def _solve_and_jacobian(g, single=False):
    h, vp, vs, rho = (np.ascontiguousarray(g[k]) for k in ("thickness", "vp", "vs", "rho"))
    periods = np.asarray(g["periods"], dtype=np.float64)
    nm, wave = int(g["nmodes"]), int(g["wave"])
    B, L = h.shape
    eng = _engine(B, L, periods.size, nm, single)
    try:
        out = eng.run(h, vp, vs, rho, periods, None, 1e-12, 1., wave, group=True)
        jc, ju, failed = eng.jacobian(h, vp, vs, rho, periods, wave, out["velocity"], out["group_velocity"])
    finally:
        eng.close()
    return (h, vp, vs, rho), periods, wave, out, jc, ju, failed


def _row_err(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize("name", ["jac_config4_rayleigh", "jac_config4_love", "jac_water_rayleigh"])
@pytest.mark.parametrize("single", [False, True])
def test_phase_jacobian_matches_reference_differences_and_oracle(name, single, oracle_lib):
    g = load_golden(name)
    model, periods, wave, out, jc, ju, failed = _solve_and_jacobian(g, single)
    v = out["velocity"]
    # the engine finds the reference's roots (masks bit-exact)
    np.testing.assert_array_equal(np.isfinite(v), np.isfinite(g["phase_velocity"]))
    assert failed == 0
    worst_fd = worst_or = 0.
    for b, m, f in zip(*np.nonzero(np.isfinite(v))):
        row = [x[b] for x in model]
        worst_fd = max(worst_fd, _row_err(jc[b, m, f], g["jac_phase_fd"][b, m, f]))
        ref = oracle_lib.phase_jacobian(*row, periods[f], v[b, m, f], wave)
        worst_or = max(worst_or, _row_err(jc[b, m, f], ref))
    assert worst_fd < PHASE_TOL_FD, worst_fd
    assert worst_or < PHASE_TOL_ORACLE, worst_or
    # missing roots give NaN rows
    assert np.isnan(jc[~np.isfinite(v)]).all()


@pytest.mark.parametrize("name", ["jac_config4_rayleigh", "jac_config4_love", "jac_water_rayleigh"])
def test_group_jacobian_matches_differences_of_oracle_group_velocity(name, oracle_lib):
    g = load_golden(name)
    model, periods, wave, out, jc, ju, failed = _solve_and_jacobian(g)
    v, u = out["velocity"], out["group_velocity"]
    cells = list(zip(*np.nonzero(np.isfinite(u))))
    assert cells
    worst = 0.
    for b, m, f in cells[::5]:  # a fifth of the roots: each needs 2 x 4L polished group velocities
        row = [x[b] for x in model]
        ref = oracle_lib.group_jacobian_fd(*row, periods[f], v[b, m, f], wave)
        worst = max(worst, _row_err(ju[b, m, f], ref))
    assert worst < GROUP_TOL_FD, worst
    # a missing group velocity gives a NaN group row
    assert np.isnan(ju[~np.isfinite(u)]).all()


def test_vjp_is_the_weighted_sum_of_the_jacobians():
    g = load_golden("jac_config4_rayleigh")
    model, periods, wave, out, jc, ju, _ = _solve_and_jacobian(g)
    h = model[0]
    B, L = h.shape
    rng = np.random.default_rng(5)
    wc = rng.normal(size=out["velocity"].shape)
    wu = rng.normal(size=out["velocity"].shape)
    eng = _engine(B, L, periods.size, int(g["nmodes"]))
    try:
        grad = eng.vjp(*model, periods, wave, out["velocity"], wc, wu, out["group_velocity"])
        grad_c = eng.vjp(*model, periods, wave, out["velocity"], wc, None, out["group_velocity"])
    finally:
        eng.close()
    fin_c = np.isfinite(out["velocity"])
    fin_u = np.isfinite(out["group_velocity"])
    jcz = np.where(fin_c[..., None, None], jc, 0.)
    juz = np.where(fin_u[..., None, None], ju, 0.)
    expect = np.einsum("bmt,bmtpl->pbl", wc, jcz) + np.einsum("bmt,bmtpl->pbl", wu, juz)
    expect_c = np.einsum("bmt,bmtpl->pbl", wc, jcz)
    scale = np.abs(expect).max()
    assert np.abs(grad - expect).max() < 1e-12 * scale
    assert np.abs(grad_c - expect_c).max() < 1e-12 * np.abs(expect_c).max()


def test_jacobians_match_differences_of_the_engines_own_fp64_solver():
    """Central differences (1e-6 relative) of the plain FP64 engine's roots and group
    velocities, at c_tol_rel 1e-13, on two config-4 models."""
    g = load_golden("jac_config4_rayleigh")
    model, periods, wave, out, jc, ju, _ = _solve_and_jacobian(g)
    B, L = model[0].shape
    b = 1
    base = [x[b].copy() for x in model]
    perturbed, index = [], []
    for p in range(4):
        for j in range(L):
            if base[p][j] == 0.:
                continue
            for sgn in (1., -1.):
                m = [x.copy() for x in base]
                m[p][j] *= 1. + sgn * 1e-6
                perturbed.append(m)
            index.append((p, j))
    batch = [np.stack([r[i] for r in perturbed]) for i in range(4)]
    eng = _engine(len(perturbed), L, periods.size, int(g["nmodes"]))
    try:
        res = eng.run(*batch, periods, None, 1e-13, 1., wave, group=True)
    finally:
        eng.close()
    fc = np.zeros(jc.shape[1:])
    fu = np.zeros(jc.shape[1:])
    for n, (p, j) in enumerate(index):
        step = 2e-6 * base[p][j]
        fc[:, :, p, j] = (res["velocity"][2 * n] - res["velocity"][2 * n + 1]) / step
        fu[:, :, p, j] = (res["group_velocity"][2 * n] - res["group_velocity"][2 * n + 1]) / step
    worst_c = worst_u = 0.
    for m, f in zip(*np.nonzero(np.isfinite(out["group_velocity"][b]))):
        worst_c = max(worst_c, _row_err(jc[b, m, f], fc[m, f]))
        worst_u = max(worst_u, _row_err(ju[b, m, f], fu[m, f]))
    assert worst_c < 1e-6, worst_c
    assert worst_u < 1e-5, worst_u


def test_autograd_misfit_gradient():
    """Gradient of the L2 misfit against a perturbed target through
    torch.autograd equals central differences of the misfit."""
    import torch
    from modisp_b200 import autograd, workloads
    batch, periods, nmodes = workloads.config4(8)
    dev = torch.device("cuda", 0)
    B, L = batch["thickness"].shape
    t = {k: torch.tensor(batch[k], dtype=torch.float64, device=dev) for k in batch}
    rng = np.random.default_rng(3)
    target = {k: torch.tensor(batch[k] * (1. + .01 * rng.normal(size=batch[k].shape)), dtype=torch.float64,
                              device=dev) for k in batch}
    solver = autograd.DifferentiableSolver(B, L, periods, nmodes, precision="mixed", c_tol_rel=1e-12)
    try:
        with torch.no_grad():
            obs_c, obs_u = solver(target["thickness"], target["vp"], target["vs"], target["rho"])
        params = {k: v.clone().requires_grad_(True) for k, v in t.items()}
        c, u = solver(params["thickness"], params["vp"], params["vs"], params["rho"])
        loss = autograd.misfit(c, u, obs_c, obs_u)
        loss.backward()
        grads = {k: params[k].grad.cpu().numpy() for k in params}

        def loss_at(values):
            with torch.no_grad():
                cc, uu = solver(values["thickness"], values["vp"], values["vs"], values["rho"])
                return float(autograd.misfit(cc, uu, obs_c, obs_u))

        checked = 0
        for key, b, j in (("vs", 0, 2), ("vp", 1, 5), ("rho", 2, 7), ("thickness", 3, 1), ("vs", 4, L - 1)):
            x0 = float(t[key][b, j])
            step = 1e-6 * x0
            vals = []
            for sgn in (1., -1.):
                values = {k: v.clone() for k, v in t.items()}
                values[key][b, j] = x0 + sgn * step
                vals.append(loss_at(values))
            fd = (vals[0] - vals[1]) / (2 * step)
            assert abs(grads[key][b, j] - fd) <= 1e-5 * max(abs(fd), 1e-3 * np.abs(grads[key]).max()), (key, b, j)
            checked += 1
        assert checked == 5
    finally:
        solver.close()


@pytest.mark.parametrize("wave", [0, 1])
@pytest.mark.parametrize("single", [False, True])
def test_jacobians_at_the_largest_layer_count(wave, single, oracle_lib):
    """256 rows (255 thin layers over a half-space), the most the API accepts
    (python/modisp/__init__.py:152): the adjoint's checkpoints cover all 255
    layer steps, and the rows match the oracle's complex-step Jacobian."""
    L = 256
    z = np.arange(L - 1)
    vs = np.concatenate([2.0 + 2.5 * z / (L - 2), [4.7]])
    model = [np.full(L, 0.2), 1.75 * vs, vs, 1.6 + 0.3 * vs]
    model[0][-1] = 0.
    model = [np.ascontiguousarray(np.stack([x, x * (1. + 0.02 * (wave + 1))]), dtype=np.float64)
             for x in model]
    periods = np.array([4., 15., 40.])
    eng = _engine(2, L, periods.size, 2, single)
    try:
        out = eng.run(*model, periods, None, 1e-12, 1., wave, group=True)
        v = out["velocity"]
        jc, ju, failed = eng.jacobian(*model, periods, wave, v, out["group_velocity"])
    finally:
        eng.close()
    assert failed == 0
    cells = list(zip(*np.nonzero(np.isfinite(v))))
    assert len(cells) >= 8
    worst = 0.
    for b, m, f in cells:
        row = [x[b] for x in model]
        worst = max(worst, _row_err(jc[b, m, f], oracle_lib.phase_jacobian(*row, periods[f], v[b, m, f], wave)))
        assert np.isfinite(ju[b, m, f]).all()
    assert worst < PHASE_TOL_ORACLE, worst
