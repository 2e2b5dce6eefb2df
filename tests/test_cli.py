"""Command line (python -m modisp_b200): the reference's forward / check-modes /
doctor commands and NPZ keys (python/modisp/cli.py), and the ragged CSR form."""
import json

import numpy as np
import pytest

from modisp_b200.cli import main, read_model

MODEL = np.array([[.3, 2., .8, 2.], [0., 5., 2.8, 2.6]])


def test_doctor_reports_without_a_device(capsys):
    assert main(["doctor"]) == 0
    data = json.loads(capsys.readouterr().out)
    assert data["version"] == "0.5.0" and "cuda_available" in data


def test_check_modes_rejects_ragged_outputs(tmp_path):
    src = tmp_path / "ragged.npz"
    np.savez(src, layout="csr", phase_velocity=np.ones(3), periods=np.ones(3))
    with pytest.raises(ValueError, match="uniform forward output"):
        main(["check-modes", str(src), "--output", str(tmp_path / "x.npz")])


def test_ragged_inputs_reject_unsupported_options(tmp_path):
    src = tmp_path / "ragged_in.npz"
    np.savez(src, **dict(zip(["thickness", "vp", "vs", "rho"], MODEL.T)), periods=[1., 2.],
             period_offsets=[0, 2])
    with pytest.raises(ValueError, match="--cmin is not available for ragged"):
        main(["forward", str(src), "--output", str(tmp_path / "o.npz"), "--cmin", "1"])
    model, periods, offsets, modes = read_model(src)
    assert offsets.tolist() == [0, 2] and modes is None and periods.tolist() == [1., 2.]


@pytest.mark.gpu
def test_forward_and_standalone_checker(tmp_path):
    """The reference's CLI test: forward with diagnostics, then check-modes on its
    output gives the same reliability arrays."""
    src, out, check = tmp_path / "input.npz", tmp_path / "output.npz", tmp_path / "check.npz"
    np.savez(src, **dict(zip(["thickness", "vp", "vs", "rho"], MODEL.T)), periods=[1., 1.1, 1.2])
    assert main(["forward", str(src), "--output", str(out), "--wave", "love", "--refinement", "chandrupatla",
                 "--close-root-rtol", "0.02", "--check-continuity"]) == 0
    assert main(["check-modes", str(out), "--output", str(check)]) == 0
    with np.load(out) as z, np.load(check) as c:
        assert str(z["refinement"]) == "chandrupatla" and str(z["love_strategy"]) == "phase"
        assert z["phase_velocity"].shape[2] == 3 and np.isfinite(z["phase_velocity"]).any()
        for key in c.files:
            forward_key = "mode_reliability_flags" if key == "continuity_flags" else key
            np.testing.assert_array_equal(z[forward_key], c[key])


@pytest.mark.gpu
def test_forward_ragged_matches_the_ragged_api(tmp_path):
    from modisp_b200 import workloads
    from modisp_b200.ragged import dispersion_ragged
    batch = workloads.crustal_batch(12, workloads.SEED + 9)
    rng = np.random.default_rng(3)
    per = [np.geomspace(rng.uniform(.3, 2.), rng.uniform(5., 40.), rng.integers(3, 12)) for _ in range(12)]
    offsets = np.concatenate([[0], np.cumsum([p.size for p in per])])
    modes = rng.integers(1, 6, 12)
    src, out = tmp_path / "ragged_in.npz", tmp_path / "ragged_out.npz"
    np.savez(src, **batch, periods=np.concatenate(per), period_offsets=offsets, nmodes=modes)
    assert main(["forward", str(src), "--output", str(out), "--group-velocity", "--precision", "float32"]) == 0
    want = dispersion_ragged(batch["thickness"], batch["vp"], batch["vs"], batch["rho"], per, nmodes=modes,
                             precision="mixed", group_velocity=True)
    with np.load(out) as z:
        assert str(z["layout"]) == "csr"
        np.testing.assert_array_equal(z["period_offsets"], offsets)
        np.testing.assert_array_equal(z["modes"], modes)
        np.testing.assert_array_equal(z["phase_velocity"], want.phase_velocity)
        np.testing.assert_array_equal(z["group_velocity"], want.group_velocity)
        np.testing.assert_array_equal(z["root_count"], want.root_count)
        np.testing.assert_array_equal(z["trace_flags"], want.trace_flags)
