"""The C-ABI library and the Python binding, without a GPU."""
import ctypes
import json
import re

import numpy as np
import pytest

from conftest import ROOT


def _declared_functions():
    text = (ROOT / "include" / "modisp_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(md200_\w+)\s*\(", text)))


def test_library_exports_every_declared_function():
    from modisp_b200 import _native
    lib = _native.lib()
    declared = _declared_functions()
    assert len(declared) >= 12
    for name in declared:
        assert hasattr(lib, name), name
    assert set(declared) == set(_native.EXPORTS)


def test_library_is_built_for_sm100a():
    from modisp_b200 import build
    cmd = build.command()
    assert "-gencode=arch=compute_100a,code=sm_100a" in cmd


def test_options_struct_matches_header():
    from modisp_b200 import _native
    text = (ROOT / "include" / "modisp_b200.h").read_text()
    body = text[text.index("typedef struct md200_options"):text.index("} md200_options;")]
    fields = re.findall(r"^\s*(?:int|double|long long)\s+(\w+);", body, flags=re.M)
    assert fields == [f for f, _ in _native.Options._fields_]
    o = _native.default_options()
    assert o.close_root_rtol == .005 and o.refinement == 1 and o.anchor_stride == 4


def test_no_device_is_reported_cleanly():
    from modisp_b200 import _native, plugin
    n = _native.device_count()
    assert n >= 0
    if n == 0:
        assert not plugin.available(0)
        with pytest.raises(RuntimeError):
            _native.Engine(0, 4, 3, 2, 1, _native.default_options())
        assert "CUDA" in _native.last_error() or "modisp_b200" in _native.last_error()


def test_invalid_geometry_is_rejected_before_any_device_work():
    from modisp_b200 import _native
    with pytest.raises(RuntimeError, match="invalid engine geometry"):
        _native.Engine(0, 0, 3, 2, 1, _native.default_options())
    with pytest.raises(RuntimeError, match="invalid engine geometry"):
        _native.Engine(0, 4, 300, 2, 1, _native.default_options())


def test_plugin_contract_attributes():
    import modisp_cuda
    module = modisp_cuda.load()
    assert modisp_cuda.__version__ == module.VERSION == "0.5.0"
    assert module.ABI_VERSION == 9
    for flag in ("SUPPORTS_FP32", "SUPPORTS_AUTO_ACCURACY", "SUPPORTS_CANONICAL_LOWER",
                 "SUPPORTS_GROUP_VELOCITY", "SUPPORTS_CONTINUATION"):
        assert getattr(module, flag) is True
    for fn in ("available", "set_device", "memory_info", "device_name", "qe_kernel_report",
               "love_phase_kernel_report", "_review_groups", "QeSolver"):
        assert callable(getattr(module, fn))


def test_solver_validation_matches_reference_rules():
    import modisp_b200 as md
    with pytest.raises(ValueError, match="backend"):
        md.Solver(backend="cpu")
    with pytest.raises(ValueError, match="group_rtol"):
        md.Solver(group_rtol=2.)
    with pytest.raises(ValueError, match="precision"):
        md.Solver(precision="half")
    with pytest.raises(ValueError, match="cmax must exceed cmin"):
        md.Solver(cmin=2., cmax=1.)
    from modisp_b200.api import _models
    with pytest.raises(ValueError, match="sqrt"):
        _models([1., 0.], [1., 5.], [1., 3.], [2., 2.])
    with pytest.raises(ValueError, match="water"):
        _models([1., 1., 0.], [1.5, 1.5, 5.], [0., 0., 3.], [1., 1., 2.])
    with pytest.raises(ValueError, match="256"):
        _models(np.ones(300), np.full(300, 5.), np.full(300, 3.), np.ones(300))


def test_uniform_strategy_options_follow_the_reference_rules():
    """search_strategy="uniform" takes the reference's constructor rules
    (python/modisp/__init__.py:194-217): legacy refinement and the dunkin secular
    only, no group velocity or continuation, no FP32 output, no accuracy preset;
    its accuracy label is "uniform" and its tolerances the uniform defaults."""
    import modisp_b200 as md
    s = md.Solver(search_strategy="uniform")
    assert (s.accuracy, s.refinement, s.c_tol_rel, s.sampling_rtol) == ("uniform", "legacy", 1e-6, 1e-3)
    assert md.Solver(search_strategy="uniform", accuracy="auto").accuracy == "uniform"
    for kwargs, err in ((dict(group_velocity=True), NotImplementedError),
                        (dict(frequency_strategy="anchor_continuation"), NotImplementedError),
                        (dict(refinement="brent"), NotImplementedError),
                        (dict(secular="fast"), NotImplementedError),
                        (dict(precision="float32"), ValueError),
                        (dict(accuracy="high"), ValueError),
                        (dict(adaptive_period_threshold=1.), ValueError)):
        with pytest.raises(err):
            md.Solver(search_strategy="uniform", **kwargs)
    from modisp_b200 import legacy
    with pytest.raises(ValueError, match="nc must be at least 3"):
        legacy.UniformSolver(nc=2)
    with pytest.raises(ValueError, match="cmin must be positive"):
        legacy.UniformSolver(cmin=0.)
    # input checks of the legacy solver (python/modisp/_legacy.py:224-290), before any device work
    u = legacy.UniformSolver()
    h, vp, vs, rho = [1., 0.], [3., 5.], [1.5, 2.8], [2., 2.5]
    for args, match in ((([1., 0.], [1.4, 5.], vs, rho), "vp must exceed vs"),
                        (([-1., 0.], vp, vs, rho), "non-negative"),
                        ((h, vp, [0., 2.8], rho), "vs must be positive"),
                        ((h, vp, vs, [2., np.nan]), "rho must be finite"),
                        (([1.], [3.], [1.5], [2.]), "at least 2 layers")):
        with pytest.raises(ValueError, match=match):
            u(*args, [1.])
    with pytest.raises(ValueError, match="periods must be positive"):
        u(h, vp, vs, rho, [0.])
    with pytest.raises(ValueError, match="above the largest half-space Vs"):
        legacy.UniformSolver(cmax=3.)(h, vp, vs, rho, [1.])


def test_workloads_have_the_stated_shapes():
    from modisp_b200 import workloads
    batch, periods, nmodes = workloads.config2(64)
    assert batch["thickness"].shape == (64, 21) and periods.size == 60 and nmodes == 5
    assert np.all(batch["thickness"][:, -1] == 0.)
    real = (batch["thickness"] > 0).sum(axis=1)
    assert real.min() >= 8 and real.max() <= 20
    assert np.all(batch["vp"] / batch["vs"] > 1.69)
    lvz, _, _ = workloads.config3(200)
    drops = np.any(lvz["vs"][:, 1:-1] < 0.81 * lvz["vs"][:, :-2], axis=1)
    assert 0.15 < drops.mean() < 0.45
    b4, p4, k4 = workloads.config4(16)
    assert b4["thickness"].shape == (16, 13) and p4.size == 40 and k4 == 3


def test_ragged_layout_and_validation():
    """CSR bookkeeping of the ragged API (no GPU needed)."""
    from modisp_b200.ragged import RaggedDispersion, _csr
    off, flat = _csr([np.array([1., 2.]), np.array([3.]), np.array([])], 3)
    assert off.tolist() == [0, 2, 3, 3] and flat.tolist() == [1., 2., 3.]
    with pytest.raises(ValueError):
        _csr([np.array([1.])], 2)
    with pytest.raises(ValueError):
        _csr([np.array([-1.]), np.array([2.])], 2)
    with pytest.raises(ValueError):
        _csr((np.array([0, 2, 1]), np.array([1., 2.])), 2)
    modes = np.array([2, 1, 3])
    cells = modes * np.diff(off)
    outb = np.concatenate([[0], np.cumsum(cells)[:-1]])
    vel = np.arange(cells.sum(), dtype=float)
    r = RaggedDispersion(off, flat, modes, outb, vel, np.zeros(3, np.uint32), np.zeros(3, np.int32),
                         np.array([2, 2, 1]), None, None, "rayleigh", {})
    assert r.phase_velocity_of(0).tolist() == [[0., 1.], [2., 3.]]
    assert r.phase_velocity_of(1).tolist() == [[4.]]
    assert r.phase_velocity_of(2).shape == (3, 0)
    assert r.root_count_of(0).tolist() == [2, 2]


def test_autotuner_picks_the_fastest_shape_and_caches_it(tmp_path, monkeypatch):
    """Search, identity check and cache of the launch-shape autotuner (fake timer, no GPU)."""
    from modisp_b200 import autotune
    monkeypatch.setenv("MODISP_B200_CACHE", str(tmp_path))
    sample = {k: np.ones((4, 6)) for k in ("thickness", "vp", "vs", "rho")}
    same = {"velocity": np.arange(6.), "counts": np.arange(3), "flags": np.zeros(3, np.uint32)}
    calls = []

    def timer(shape, *args):
        calls.append(shape)
        return {(2, 0, 2): 1.0}.get(tuple(shape), 2.0), same

    best = autotune.autotune(sample, [1., 2.], 3, 0, True, timer=timer)
    assert best == (2, 0, 2) and len(calls) == len(autotune.CANDIDATES)
    assert {c[2] for c in autotune.CANDIDATES} == {0, 1, 2}  # both scan forms and the automatic choice
    assert {c[2] for c in autotune.candidates(False)} == {0}  # the FP64 engine has one scan form
    table = json.loads(autotune.cache_path().read_text())
    assert list(table.values())[0]["shape"] == [2, 0, 2]
    calls.clear()
    assert autotune.autotune(sample, [1., 2.], 3, 0, True, timer=timer) == (2, 0, 2) and not calls  # cached
    from modisp_b200 import _native
    o = _native.Options()
    autotune.apply(o, (2, 3, 1))
    assert (o.warps_per_block, o.blocks_per_sm, o.scan_mode) == (2, 3, 1)

    def bad_timer(shape, *args):
        out = dict(same, velocity=same["velocity"] + (shape[0] == 1))
        return 1.0, out

    with pytest.raises(RuntimeError, match="changed"):
        autotune.autotune(sample, [1., 2., 3.], 3, 0, True, timer=bad_timer, use_cache=False)


def test_header_compiles_as_c_and_plan_layout_matches(tmp_path):
    """The C ABI header is plain C99, and md200_period_plan has the field offsets
    and size of the numpy dtype the Python layer fills."""
    import shutil
    import subprocess
    from modisp_b200 import _native
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    src = tmp_path / "layout.c"
    src.write_text('#include <stddef.h>\n#include <stdio.h>\n#include "modisp_b200.h"\n'
                   'int main(void) { printf("%zu %zu %zu %zu %zu %zu\\n", sizeof(md200_period_plan), '
                   'offsetof(md200_period_plan, older), offsetof(md200_period_plan, kind), '
                   'offsetof(md200_period_plan, dup_begin), offsetof(md200_period_plan, dup_end), '
                   'offsetof(md200_period_plan, ratio)); return 0; }\n')
    exe = tmp_path / "layout"
    subprocess.run([cc, "-std=c99", "-Wall", "-Werror", "-pedantic", f"-I{ROOT / 'include'}", str(src), "-o",
                    str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    dt = _native.PERIOD_PLAN
    assert got == [dt.itemsize, dt.fields["older"][1], dt.fields["kind"][1], dt.fields["dup_begin"][1],
                   dt.fields["dup_end"][1], dt.fields["ratio"][1]]
