"""md200_group_roots_static, the allocation-free review-group entry point.

Some callers of the group-velocity bridge cannot call cudaMalloc: code whose GPU
memory is owned by another allocator (a framework's caching allocator that has
reserved the device), and repair loops that must not pay cudaFree's device-wide
synchronisation on every trace.  This entry point keeps its scratch in a static
16 KiB device array instead; its results must equal those of the allocating
md200_group_roots.  Both are called through the C ABI, twice in a row on different
traces (the second call must not see the first call's leftovers).
"""
import ctypes

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def _call(name, fn, case, b, f):
    from modisp_b200 import _native
    lib = _native.lib()
    g = load_golden(case)
    model = [np.ascontiguousarray(g[k][b], dtype=np.float64) for k in ("thickness", "vp", "vs", "rho")]
    v = g["phase_velocity"][b, :, f]
    roots = np.ascontiguousarray(v[np.isfinite(v)])
    modes = int(g["nmodes"]) + 1  # one slot past the roots: a missing root too
    group = np.full(modes, -1.)
    flags = np.full(modes, 12345, dtype=np.uint32)
    status = getattr(lib, fn)(*(_native.ptr(a) for a in model), model[0].size, int(g["wave"]),
                              float(g["periods"][f]), _native.ptr(roots), roots.size, modes, .005,
                              _native.ptr(group), _native.ptr(flags))
    assert status == 0, _native.last_error()
    return group, flags


@pytest.mark.parametrize("case,b,f", [("ref_crustal48_rayleigh", 3, 10), ("ref_lvz48_love", 7, 30)])
def test_static_scratch_matches_allocating_entry_point(case, b, f):
    # two consecutive calls of the static variant (this case, then another trace)
    g_static, f_static = _call(case, "md200_group_roots_static", case, b, f)
    g_other, _ = _call(case, "md200_group_roots_static", case, (b + 5) % 48, (f + 17) % 60)
    g_alloc, f_alloc = _call(case, "md200_group_roots", case, b, f)
    np.testing.assert_array_equal(f_static, f_alloc)
    finite = np.isfinite(g_alloc)
    assert finite.sum() >= 2
    np.testing.assert_allclose(g_static[finite], g_alloc[finite], rtol=1e-12)
    assert np.all(np.isnan(g_static[~finite]))
    # and again after the other trace used the same scratch
    g_again, f_again = _call(case, "md200_group_roots_static", case, b, f)
    np.testing.assert_array_equal(f_again, f_alloc)
    np.testing.assert_allclose(g_again[finite], g_alloc[finite], rtol=1e-12)
    other = g_other[np.isfinite(g_other)]
    if other.size:  # the interleaved call really wrote different values into the scratch
        assert other[0] != g_again[finite][0]


@pytest.mark.parametrize("fn", ["md200_group_roots_static", "md200_group_roots"])
def test_nan_and_negative_packed_roots_are_missing_roots(fn):
    """A packed root that is NaN or not positive is a missing root (the reference's
    group_velocity, cpp/common/group_velocity.hpp:31), in both entry points."""
    from modisp_b200 import _native
    lib = _native.lib()
    g = load_golden("ref_crustal48_rayleigh")
    b, f = 3, 10
    model = [np.ascontiguousarray(g[k][b], dtype=np.float64) for k in ("thickness", "vp", "vs", "rho")]
    v = g["phase_velocity"][b, :, f]
    good = v[np.isfinite(v)]
    assert good.size >= 4
    # (a root right below a negative one would count as a close pair, as in the
    # reference's close-root rule, so the negative root comes first)
    roots = np.ascontiguousarray(np.array([-1.0, good[0], np.nan, good[2], good[3]]))
    modes = roots.size
    group = np.full(modes, -1.)
    flags = np.full(modes, 12345, dtype=np.uint32)
    status = getattr(lib, fn)(*(_native.ptr(a) for a in model), model[0].size, int(g["wave"]),
                              float(g["periods"][f]), _native.ptr(roots), roots.size, modes, .005,
                              _native.ptr(group), _native.ptr(flags))
    assert status == 0, _native.last_error()
    np.testing.assert_array_equal(flags[[0, 2]], [1, 1])  # GROUP_MISSING_ROOT
    assert np.all(np.isnan(group[[0, 2]]))
    assert np.all(flags[[1, 3, 4]] == 0) and np.all(np.isfinite(group[[1, 3, 4]]))


def test_requests_beyond_the_static_scratch_are_rejected():
    from modisp_b200 import _native
    lib = _native.lib()
    L, known, modes = 256, 200, 200  # 7*256 + 200 + 200 + 100 doubles > 2048
    model = [np.ascontiguousarray(x) for x in (np.full(L, .5), np.full(L, 6.), np.full(L, 3.5), np.full(L, 2.7))]
    roots = np.linspace(1., 3., known)
    group = np.zeros(modes)
    flags = np.zeros(modes, dtype=np.uint32)
    status = lib.md200_group_roots_static(*(_native.ptr(a) for a in model), L, 0, 1.0, _native.ptr(roots), known,
                                          modes, .005, _native.ptr(group), _native.ptr(flags))
    assert status != 0
    assert "static scratch" in _native.last_error()
