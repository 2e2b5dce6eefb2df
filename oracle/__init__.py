"""The oracle: CPU checkers for the modisp_b200 CUDA engine.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline / reference legs of ``bench.py`` import this package, and only to
check or time against it.  The product package ``modisp_b200`` never imports it.

Two checkers live here:

* ``libmdoracle.so`` (``md_oracle.c``): a C restatement of the reference's FP64
  numerics -- secular functions, search window, Brent refinement, a dense-grid
  root search -- plus complex-step derivatives in long double for group
  velocities and Jacobians.
* ``_ref/_cpu*.so``: the reference's own CPU engine (``CpuSolver``), compiled
  from its unmodified sources by ``oracle/Makefile``.  It is the root-set
  oracle: mode counts, labels and masks are compared against it.

Build both with ``make -C oracle`` (``__graft_entry__.build()`` does this).
"""
from __future__ import annotations

import ctypes
import glob
import importlib.util
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_LIB = None
_REF = None

TWO_PI = 6.283185307179586476925286766559


def build(quiet: bool = True) -> None:
    """Compile the C restatement and, where the reference tree exists, the reference engine."""
    import subprocess
    cmd = ["make", "-C", str(HERE), "all"]
    subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL if quiet else None)


def lib():
    """ctypes handle of the C restatement (builds it on first use)."""
    global _LIB
    if _LIB is None:
        path = HERE / "_build" / "libmdoracle.so"
        if not path.exists():
            build()
        L = ctypes.CDLL(str(path))
        d = ctypes.c_double
        P = ctypes.POINTER(ctypes.c_double)
        i = ctypes.c_int
        L.mdo_secular.restype = d
        L.mdo_secular.argtypes = [P, P, P, P, i, i, d, d, P]
        L.mdo_love_phase.restype = d
        L.mdo_love_phase.argtypes = [P, P, P, i, d, d]
        L.mdo_bounds.restype = None
        L.mdo_bounds.argtypes = [P, P, P, P, i, i, P, P]
        L.mdo_refine.restype = d
        L.mdo_refine.argtypes = [P, P, P, P, i, i, d, d, d, d, d, d, ctypes.POINTER(i)]
        L.mdo_dense_roots.restype = i
        L.mdo_dense_roots.argtypes = [P, P, P, P, i, i, d, d, d, i, d, P]
        L.mdo_derivatives.restype = None
        L.mdo_derivatives.argtypes = [P, P, P, P, i, i, d, d, P, P]
        L.mdo_group.restype = i
        L.mdo_group.argtypes = [P, P, P, P, i, i, d, d, d, d, P]
        L.mdo_parameter_derivatives.restype = None
        L.mdo_parameter_derivatives.argtypes = [P, P, P, P, i, i, d, d, P, P]
        L.mdo_uniform_refine.restype = None
        V = ctypes.c_void_p
        L.mdo_uniform_refine.argtypes = [V, i, P, P, P, P, i, ctypes.c_float, i, d, d, d, d, P, V, V]
        _LIB = L
    return _LIB


def reference():
    """The reference's compiled CPU engine module (``_cpu``), or None if not built."""
    global _REF
    if _REF is None:
        hits = sorted(glob.glob(str(HERE / "_ref" / "_cpu*.so")))
        if not hits:
            return None
        spec = importlib.util.spec_from_file_location("_cpu", hits[0])
        module = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(module)
        _REF = module
    return _REF


_WRAPPER = None
_CUDA = None


def reference_wrapper():
    """The reference's own Python package (``modisp``), unmodified, as the oracle
    recipe stages it under ``_ref/modisp`` with the reference CPU engine as its
    ``_cpu``; None where it is not staged.  Its loader finds this repository's
    ``modisp_cuda`` package for ``backend="cuda"``."""
    global _WRAPPER
    if _WRAPPER is None:
        root = HERE / "_ref"
        engine = reference()
        if engine is None or not (root / "modisp" / "__init__.py").is_file():
            return None
        import sys
        # one loaded copy of the engine serves both the wrapper (its `from . import
        # _cpu`) and reference(): a pybind11 module cannot be loaded twice
        sys.modules.setdefault("modisp._cpu", engine)
        if str(root) not in sys.path:
            sys.path.insert(0, str(root))
        import modisp
        _WRAPPER = modisp
    return _WRAPPER


def reference_cuda():
    """The reference's own CUDA plugin extension (``_cuda``), compiled for sm_100a
    from its sources by ``make -C oracle ref-cuda``; None where it is not built.
    A same-GPU comparator for bench.py, never a checker of results."""
    global _CUDA
    if _CUDA is None:
        hits = sorted(glob.glob(str(HERE / "_ref" / "cuda" / "_cuda*.so")))
        if not hits:
            return None
        spec = importlib.util.spec_from_file_location("_cuda", hits[0])
        module = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(module)
        _CUDA = module
    return _CUDA


def _ptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _model(h, vp, vs, rho):
    arrays = [np.ascontiguousarray(x, dtype=np.float64).ravel() for x in (h, vp, vs, rho)]
    return arrays, arrays[0].size


def secular(h, vp, vs, rho, period, velocity, wave=0, shape=False):
    """F (and the shape feature g) at each velocity for one model and period."""
    (h, vp, vs, rho), L = _model(h, vp, vs, rho)
    c = np.atleast_1d(np.asarray(velocity, dtype=np.float64))
    omega = TWO_PI / period
    out = np.empty(c.size)
    g = np.empty(c.size)
    tmp = ctypes.c_double()
    for j, x in enumerate(c):
        out[j] = lib().mdo_secular(_ptr(h), _ptr(vp), _ptr(vs), _ptr(rho), L, int(wave), omega,
                                   float(x), ctypes.byref(tmp))
        g[j] = tmp.value
    return (out, g) if shape else out


def love_phase(h, vs, rho, period, velocity):
    (h, _, vs, rho), L = _model(h, h, vs, rho)
    omega = TWO_PI / period
    return np.array([lib().mdo_love_phase(_ptr(h), _ptr(vs), _ptr(rho), L, omega, float(x))
                     for x in np.atleast_1d(velocity)])


def bounds(h, vp, vs, rho, wave=0):
    """[B, 2] search windows for a [B, L] batch."""
    h, vp, vs, rho = (np.atleast_2d(np.ascontiguousarray(x, dtype=np.float64)) for x in (h, vp, vs, rho))
    out = np.empty((h.shape[0], 2))
    lo, hi = ctypes.c_double(), ctypes.c_double()
    for b in range(h.shape[0]):
        row = [np.ascontiguousarray(x[b]) for x in (h, vp, vs, rho)]
        lib().mdo_bounds(*(_ptr(r) for r in row), h.shape[1], int(wave), ctypes.byref(lo), ctypes.byref(hi))
        out[b] = lo.value, hi.value
    return out


def dense_roots(h, vp, vs, rho, period, lo, hi, K, tol=1e-12, wave=0):
    (h, vp, vs, rho), L = _model(h, vp, vs, rho)
    roots = np.full(K, np.nan)
    n = lib().mdo_dense_roots(_ptr(h), _ptr(vp), _ptr(vs), _ptr(rho), L, int(wave), float(period),
                              float(lo), float(hi), int(K), float(tol), _ptr(roots))
    return n, roots


def derivatives(h, vp, vs, rho, period, c, wave=0):
    (h, vp, vs, rho), L = _model(h, vp, vs, rho)
    fk, fw = ctypes.c_double(), ctypes.c_double()
    lib().mdo_derivatives(_ptr(h), _ptr(vp), _ptr(vs), _ptr(rho), L, int(wave), TWO_PI / period,
                          float(c), ctypes.byref(fk), ctypes.byref(fw))
    return fk.value, fw.value


def group(h, vp, vs, rho, period, root, lower, upper, wave=0):
    (h, vp, vs, rho), L = _model(h, vp, vs, rho)
    u = ctypes.c_double()
    rc = lib().mdo_group(_ptr(h), _ptr(vp), _ptr(vs), _ptr(rho), L, int(wave), TWO_PI / period,
                         float(root), float(lower), float(upper), ctypes.byref(u))
    return u.value if rc == 0 else np.nan


def parameter_derivatives(h, vp, vs, rho, period, c, wave=0):
    """(dF/dtheta [4, L] for h, vp, vs, rho; dF/dc) at one root, by complex step."""
    (h, vp, vs, rho), L = _model(h, vp, vs, rho)
    out = np.empty(4 * L)
    fc = ctypes.c_double()
    lib().mdo_parameter_derivatives(_ptr(h), _ptr(vp), _ptr(vs), _ptr(rho), L, int(wave),
                                    TWO_PI / period, float(c), _ptr(out), ctypes.byref(fc))
    return out.reshape(4, L), fc.value


def phase_jacobian(h, vp, vs, rho, period, c, wave=0):
    """dc/dtheta [4, L] (thickness, vp, vs, rho) at a root c: -F_theta / F_c from the
    long-double complex-step derivatives.  Rows of zero thickness are padding by the
    engine's convention and get 0 (as does the half-space thickness)."""
    dF, Fc = parameter_derivatives(h, vp, vs, rho, period, c, wave)
    jac = -dF / Fc
    padding = np.asarray(h, dtype=np.float64) == 0.
    padding[0] = padding[-1] = False  # the first row and the half-space are always kept
    jac[:, padding] = 0.
    jac[0, -1] = 0.
    return jac


def group_jacobian_fd(h, vp, vs, rho, period, c, wave=0, rel=1e-6, window=1e-4):
    """dU/dtheta [4, L] by central differences (relative step `rel`) of the oracle's
    polished group velocity; each perturbed root is re-polished inside
    c (1 -+ window).  Zero-valued parameters (padding thickness, fluid shear
    velocity, the half-space thickness) get 0."""
    base = [np.array(x, dtype=np.float64) for x in (h, vp, vs, rho)]
    L = base[0].size
    out = np.zeros((4, L))
    for p in range(4):
        for j in range(L):
            if base[p][j] == 0. or (p == 0 and j == L - 1):
                continue
            vals = []
            for sgn in (1., -1.):
                a = [x.copy() for x in base]
                a[p][j] *= 1. + sgn * rel
                vals.append(group(*a, period, c, c * (1. - window), c * (1. + window), wave))
            out[p, j] = (vals[0] - vals[1]) / (2. * rel * base[p][j])
    return out


def reference_fd_phase_jacobian(h, vp, vs, rho, periods, nmodes, wave=0, rel=1e-6, tol=1e-13):
    """Central differences (step `rel` relative) of the reference CPU solver's roots
    for one model: (roots [nmodes, T], dc/dtheta [nmodes, T, 4, L]).  Every
    perturbed model is solved in one batched reference call; zero-valued
    parameters get 0."""
    base = [np.array(x, dtype=np.float64) for x in (h, vp, vs, rho)]
    L = base[0].size
    rows, index = [tuple(base)], []
    for p in range(4):
        for j in range(L):
            if base[p][j] == 0. or (p == 0 and j == L - 1):
                continue
            for sgn in (1., -1.):
                m = [x.copy() for x in base]
                m[p][j] *= 1. + sgn * rel
                rows.append(tuple(m))
            index.append((p, j))
    batch = [np.stack([r[i] for r in rows]) for i in range(4)]
    out = reference_solve(*batch, np.asarray(periods, dtype=np.float64), nmodes, wave=wave, tol=tol)["phase_velocity"]
    fd = np.zeros((nmodes, len(periods), 4, L))
    for n, (p, j) in enumerate(index):
        fd[:, :, p, j] = (out[1 + 2 * n] - out[2 + 2 * n]) / (2. * rel * base[p][j])
    return out[0], fd


def group_windows(roots, lower, upper, close_rtol=0.005):
    """Neighbour-midpoint windows and close-root flags (cpp/cpu/solver.cpp:96-103)."""
    n = len(roots)
    lo = np.empty(n)
    hi = np.empty(n)
    close = np.zeros(n, dtype=bool)
    for j, c in enumerate(roots):
        lo[j] = .5 * (roots[j - 1] + c) if j else lower
        hi[j] = .5 * (c + roots[j + 1]) if j + 1 < n else upper
        close[j] = (j and c - roots[j - 1] <= close_rtol * c) or (j + 1 < n and roots[j + 1] - c <= close_rtol * roots[j + 1])
    return lo, hi, close


def reference_solve(h, vp, vs, rho, periods, nmodes, wave=0, tol=1e-12, threads=None,
                    group_velocity=False, group_rtol=1e-3, accuracy=0, bounds=None):
    """Run the reference CPU engine on a [B, L] batch the way its Python wrapper does
    for ``Solver(backend="cpu", accuracy="high", search_strategy="shape_adaptive",
    secular="dunkin", refinement="brent", love_strategy="phase")``
    (python/modisp/__init__.py:343,414-424).  ``bounds`` [B, 2]: a given search
    window, run as the wrapper runs one from cmin/cmax (not automatic)."""
    ref = reference()
    if ref is None:
        raise RuntimeError("reference CPU engine not built (make -C oracle ref)")
    h, vp, vs, rho = (np.atleast_2d(np.ascontiguousarray(x, dtype=np.float64)) for x in (h, vp, vs, rho))
    periods = np.ascontiguousarray(periods, dtype=np.float64)
    threads = threads or min(256, len(os.sched_getaffinity(0)))
    automatic = bounds is None
    bnd = ref.bounds(h, vp, vs, rho, int(wave), None, None) if automatic else np.ascontiguousarray(bounds, np.float64)
    solver = ref.CpuSolver(int(threads), int(accuracy), 0., .005, True, .001, 0, 1, 1)
    out = solver.run(h, vp, vs, rho, periods, bnd, int(nmodes), int(wave), automatic, float(tol), 1.,
                     False, bool(group_velocity), float(group_rtol), True)
    velocity, flags, stats, levels, counts, extras = out
    counts = counts.copy()
    counts[(flags & 4) != 0] = -1
    return dict(phase_velocity=velocity, trace_flags=flags, stats=stats, search_level=levels,
                root_count=counts, group_velocity=extras["group_velocity"],
                group_velocity_flags=extras["group_velocity_flags"], search_bounds=bnd)


def uniform_refine(rows, h, vp, vs, rho, periods, nmodes, cmin, cmax, c_tol_rel=1e-6, f_accept=1.0):
    """Stage 2 of the legacy uniform path (cpp/cuda/refine.cuh:131-317) on given
    stage 1 values ``rows`` [B, T, nc] (float32): velocity [B, nmodes, T], trace
    flags [B, T] and the six counters, computed trace by trace on the CPU."""
    rows = np.ascontiguousarray(rows, dtype=np.float32)
    h, vp, vs, rho = (np.atleast_2d(np.ascontiguousarray(x, dtype=np.float64)) for x in (h, vp, vs, rho))
    B, T, nc = rows.shape
    per = np.asarray(periods, dtype=np.float32)
    out = np.full((B, nmodes, T), np.nan)
    flags = np.zeros((B, T), np.uint32)
    stats = np.zeros(6, np.uint64)
    o = np.empty(nmodes)
    fl = np.zeros(1, np.uint32)
    for b in range(B):
        row_args = [np.ascontiguousarray(x[b]) for x in (h, vp, vs, rho)]
        for t in range(T):
            fl[0] = 0
            lib().mdo_uniform_refine(rows[b, t].ctypes.data, nc, *(_ptr(x) for x in row_args), h.shape[1],
                                     float(per[t]), int(nmodes), float(cmin), float(cmax), float(c_tol_rel),
                                     float(f_accept), _ptr(o), fl.ctypes.data, stats.ctypes.data)
            out[b, :, t] = o
            flags[b, t] = fl[0]
    names = ("brackets", "rejected_sign", "rejected_f", "troughs", "hidden_roots", "relocated")
    return out, flags, {k: int(v) for k, v in zip(names, stats)}
