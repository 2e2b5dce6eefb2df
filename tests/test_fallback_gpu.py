"""The fallback for traces the first search could not finish.

A trace whose scan reaches the scan-point limit before it holds all its brackets,
or that meets a non-finite value, is re-scanned in FP64 with a 16x larger limit
(the reference escalates such traces to its adaptive ladder and dense grid,
cpp/cpu/solver.cpp:254-370,517-584).  The test lowers the first search's limit
(option scan_points) far below what the traces need, so every long trace goes
through the fallback; the results must still be the reference's, and equal the
plain FP64 engine's bit for bit on those traces.
"""
import numpy as np
import pytest

from conftest import load_golden
from test_parity_gpu import assert_root_parity, ENGINE_TOL

pytestmark = pytest.mark.gpu


def solve(g, single, **opts):
    from modisp_b200 import _native
    h = g["thickness"]
    o = _native.default_options()
    o.single_precision, o.group_velocity = int(single), 1
    for k, v in opts.items():
        setattr(o, k, v)
    e = _native.Engine(0, h.shape[0], h.shape[1], g["periods"].size, int(g["nmodes"]), o)
    try:
        return e.run(h, g["vp"], g["vs"], g["rho"], g["periods"], g["search_bounds"], ENGINE_TOL, 1.,
                     int(g["wave"]), group=True)
    finally:
        e.close()


@pytest.mark.parametrize("single", [False, True], ids=["fp64", "fp32scan"])
@pytest.mark.parametrize("name", ["ref_crustal48_rayleigh", "ref_lvz48_love", "ref_deep4_k100_rayleigh"])
def test_unfinished_traces_are_rescanned(name, single):
    g = load_golden(name)
    capped = solve(g, single, scan_points=48)
    assert_root_parity(g, capped, f"{name} capped")
    fell = (capped["flags"] & 8192) != 0
    assert fell.sum() > 0 and capped["stats"]["fallback_rescans"] == int(fell.sum())
    np.testing.assert_array_equal(capped["levels"][fell], 24)
    assert not np.any(capped["flags"] & 4)
    # the fallback is the FP64 scan with a larger limit: its traces equal the plain FP64 engine's
    plain = solve(g, False)
    v, p = capped["velocity"].view(np.uint64), plain["velocity"].view(np.uint64)
    for b, f in zip(*np.nonzero(fell)):
        np.testing.assert_array_equal(v[b, :, f], p[b, :, f])
        np.testing.assert_array_equal(capped["group_velocity"][b, :, f].view(np.uint64),
                                      plain["group_velocity"][b, :, f].view(np.uint64))
    assert capped["stats"]["roots"] == int(np.isfinite(capped["velocity"]).sum())
