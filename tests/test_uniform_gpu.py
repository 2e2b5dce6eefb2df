"""The legacy uniform-grid path (search_strategy="uniform") on the GPU.

Checked against the reference's own implementation of it -- its CUDA stages
(cpp/cuda/coarse_scan.cu, cpp/cuda/refine.cu) run by
tests/golden/make_uniform_golden.py into the committed ``uniform_*`` fixtures -- and
against the oracle's CPU restatement of stage 2 (oracle/md_oracle.c,
mdo_uniform_refine), which tests/test_oracle.py pins to the same fixtures:

* stage 2 on the reference's own stage 1 values returns the reference's roots bit
  for bit, with its trace flags and counters;
* stage 1 values agree with the reference's in sign wherever |F| > 1e-3 and
  single precision resolves them (velocities at or above max(vs) / 16: below that the reference's
  standard single-precision recurrence loses the sign of deep evanescent layers,
  the ``lowc6`` case);
* the whole path on its own values returns the oracle's roots on those values,
  and the reference's roots on the cases whose scan stays above max(vs) / 16;
* the reference's unmodified Python wrapper runs the path through this
  repository's plugin (``Solver(backend="cuda", search_strategy="uniform")`` and
  its ``_legacy.Solver``), and modisp_b200.Solver returns the same batch.
"""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

CASES = ["crustal12", "lvz12", "lowc6", "deep4"]
RESOLVED = ["crustal12", "lvz12", "deep4"]  # scans that stay at or above max(vs) / 16


def _golden(case):
    g = load_golden(f"uniform_{case}")
    g["names"] = [str(x) for x in g["stat_names"]]
    return g


def _model(g):
    return [np.ascontiguousarray(g[k]) for k in ("thickness", "vp", "vs", "rho")]


def _stages(g):
    from modisp_b200 import plugin
    model = _model(g)
    B, L = model[0].shape
    scan, refine = plugin.CoarseScan(B, L), plugin.Refine(B, L)
    for stage in (scan, refine):
        stage.upload_models(*model)
        stage.upload_periods(g["periods"])
    scan.allocate(int(g["nc"]))
    refine.allocate(int(g["nc"]), int(g["nmodes"]))
    return scan, refine


def _run(g, rows=None):
    scan, refine = _stages(g)
    cmin, cmax = float(g["cmin"]), float(g["cmax"])
    if rows is None:
        scan.run(cmin, cmax)
    else:  # the reference's stage 1 values in place of this scan's
        scan._u.set_rows(rows, cmin, cmax)
        scan._range = (cmin, cmax)
    refine.run(scan, cmin, cmax, float(g["c_tol_rel"]), float(g["f_accept"]), int(g["nmodes"]))
    out = scan.download() if rows is None else None, refine.download(), refine.flags(), refine.stats()
    scan.close()
    refine.close()
    return out


def _same_roots(v, ref):
    np.testing.assert_array_equal(np.isfinite(v), np.isfinite(ref))
    m = np.isfinite(ref)
    np.testing.assert_array_equal(v[m], ref[m])


@pytest.mark.parametrize("case", CASES)
def test_stage2_on_the_reference_values_is_the_reference(case):
    g = _golden(case)
    _, v, flags, stats = _run(g, rows=g["rows"])
    _same_roots(v, g["phase_velocity"])
    np.testing.assert_array_equal(flags, g["trace_flags"])
    assert stats == {k: int(x) for k, x in zip(g["names"], g["stats"])}


def _resolved_cells(g):
    """[B, 1, nc] mask of grid velocities at or above max(vs) / 16 of each model."""
    nc, cmin, cmax = int(g["nc"]), float(g["cmin"]), float(g["cmax"])
    c = cmin + (cmax - cmin) / (nc - 1) * np.arange(nc)
    return (c[None, :] >= g["vs"].max(axis=1)[:, None] / 16.)[:, None, :]


@pytest.mark.parametrize("case", CASES)
def test_stage1_values_agree_with_the_reference(case):
    g = _golden(case)
    rows, _, _, _ = _run(g)
    ref = g["rows"]
    np.testing.assert_array_equal(np.isnan(rows), np.isnan(ref))  # cells past the last one read
    ok = np.isfinite(ref) & np.broadcast_to(_resolved_cells(g), ref.shape)
    assert ok.sum() > 0.5 * np.isfinite(ref).sum() or case == "lowc6"
    clear = ok & (np.abs(ref) > 1e-3)
    np.testing.assert_array_equal(np.sign(rows[clear]), np.sign(ref[clear]))
    # both are single-precision values of the same max-amplitude-scaled function
    # from different operation orders; cancellation in the recurrence leaves up to
    # a few 1e-3 between them (4.2e-3 measured, on deep4)
    assert np.abs(rows[ok] - ref[ok]).max() < 1e-2


@pytest.mark.parametrize("case", CASES)
def test_whole_path_matches_the_oracle_on_its_own_values(case, oracle_lib):
    import oracle
    g = _golden(case)
    rows, v, flags, stats = _run(g)
    ov, oflags, ostats = oracle.uniform_refine(rows, *_model(g), g["periods"], int(g["nmodes"]), float(g["cmin"]),
                                               float(g["cmax"]), float(g["c_tol_rel"]), float(g["f_accept"]))
    _same_roots(v, ov)
    np.testing.assert_array_equal(flags, oflags)
    assert stats == ostats


@pytest.mark.parametrize("case", RESOLVED)
def test_whole_path_matches_the_reference(case):
    g = _golden(case)
    _, v, flags, _ = _run(g)
    _same_roots(v, g["phase_velocity"])
    np.testing.assert_array_equal(flags, g["trace_flags"])


def test_stage_errors_follow_the_reference():
    from modisp_b200 import plugin
    g = _golden("crustal12")
    model = _model(g)
    B, L = model[0].shape
    with pytest.raises(ValueError, match="must have shape"):
        plugin.CoarseScan(B, L).upload_models(model[0][:, :-1], *model[1:])
    with pytest.raises(ValueError, match="non-empty 1-D"):
        plugin.Refine(B, L).upload_periods([])
    water = [x.copy() for x in model]
    water[2][:, 0] = 0.  # a fluid top layer: not a model of this path
    with pytest.raises(RuntimeError, match="solid models"):
        plugin.CoarseScan(B, L).upload_models(*water)
    scan, refine = plugin.CoarseScan(B, L), plugin.Refine(B, L)
    with pytest.raises(RuntimeError, match="upload_models"):
        scan.run(.2, 4.)
    with pytest.raises(RuntimeError, match="allocate"):
        scan.download()
    for stage in (scan, refine):
        stage.upload_models(*model)
        stage.upload_periods(g["periods"])
    with pytest.raises(RuntimeError, match="allocate"):
        refine.run(scan, .2, 4.)
    scan.allocate(64)
    refine.allocate(128, 3)
    with pytest.raises(ValueError, match="geometries differ"):
        refine.run(scan, .2, 4.)
    refine.allocate(64, 3)
    with pytest.raises(ValueError, match="has not been run"):
        refine.run(scan, .2, 4.)
    scan.run(.2, 4.)
    with pytest.raises(ValueError, match="ranges differ"):
        refine.run(scan, .2, 4.5)
    with pytest.raises(RuntimeError, match="exceeds the allocated"):
        refine.run(scan, .2, 4., nmodes=4)
    refine.run(scan, .2, 4., nmodes=2)
    assert refine.download().shape == (B, 2, g["periods"].size)
    assert "regs=" in scan.kernel_report() and "regs=" in refine.kernel_report()
    assert set(refine.stats()) == set(plugin.STAT_NAMES)


@pytest.fixture(scope="module")
def modisp():
    import oracle
    wrapper = oracle.reference_wrapper()
    if wrapper is None:
        pytest.skip("reference wrapper not staged (make -C oracle REFERENCE=<checkout>)")
    return wrapper


def test_reference_wrapper_runs_the_uniform_path_on_the_plugin(modisp):
    """The reference's own facade check (its tests/test_api.py uniform case) through
    this plugin, then the fixture: the wrapper's defaults (nc 512, c_tol_rel 1e-6,
    cmax the largest half-space vs) are the fixture's settings."""
    from modisp._legacy import Solver as Legacy
    g = _golden("crustal12")
    h, vp, vs, rho = _model(g)
    per = g["periods"]
    with Legacy(search_strategy="uniform", cmin=.2) as old:
        expected = old(h, vp, vs, rho, per, nmodes=5)
    with modisp.Solver(backend="cuda", search_strategy="uniform", cmin=.2) as new:
        result = new(h, vp, vs, rho, per, nmodes=5)
    assert result.backend_used == "cuda" and result.secular == "dunkin"
    np.testing.assert_array_equal(result.phase_velocity, expected.phase_velocity)
    np.testing.assert_array_equal(result.trace_flags & 255, expected.trace_flags)
    _same_roots(result.phase_velocity, g["phase_velocity"])
    np.testing.assert_array_equal(result.trace_flags & 255, g["trace_flags"])
    assert (result.search_level == -2).all()

    import modisp_b200
    with modisp_b200.Solver(search_strategy="uniform", cmin=.2) as ours:
        mine = ours(h, vp, vs, rho, per, nmodes=5)
    np.testing.assert_array_equal(mine.phase_velocity, result.phase_velocity)
    np.testing.assert_array_equal(mine.trace_flags, result.trace_flags)
    np.testing.assert_array_equal(mine.root_count, result.root_count)
    np.testing.assert_array_equal(mine.search_level, result.search_level)
    np.testing.assert_array_equal(mine.search_bounds, result.search_bounds)
    assert mine.accuracy == result.accuracy == "uniform"
