"""The legacy uniform-grid Rayleigh path (``search_strategy="uniform"``).

The reference serves it through ``python/modisp/_legacy.py:124-431`` (a FP32
scan on a uniform velocity grid, then FP64 confirmation, trough sub-sampling
and fixed-count bisection: ``cpp/cuda/coarse_scan.cuh``, ``cpp/cuda/refine.cuh``)
and wraps it in ``Solver`` at ``python/modisp/__init__.py:302-311``.  Here the
two stages are the plugin classes ``CoarseScan`` and ``Refine`` over the
engine's ``md200_uniform_*`` kernels; this module holds the input checks and
the stage calls of the legacy solver, with its error messages.
"""
from __future__ import annotations

import numpy as np

# trace flags of the legacy path (cpp/cuda/refine.cuh:58-64)
TRACE_UNRESOLVED_BRACKET = 1 << 0
TRACE_RELOCATED = 1 << 1


def _as_2d(x, name, B=None):
    a = np.ascontiguousarray(x, dtype=np.float64)
    if a.ndim == 1:
        a = a[None, :]
    if a.ndim != 2:
        raise ValueError(f"{name} must be [B, L] or [L], got shape {a.shape}")
    if B is not None and a.shape[0] != B:
        raise ValueError(f"{name} has {a.shape[0]} models but the batch has {B}; all of "
                         f"thickness/vp/vs/rho must agree")
    return a


class UniformSolver:
    """Reusable stage objects for one geometry (python/modisp/_legacy.py:124-350).

    ``__call__`` validates a solid Rayleigh batch (_legacy.py:224-290), scans it
    on ``nc`` velocities over [cmin, cmax] (cmax defaults to the batch's largest
    half-space shear velocity) and returns (velocity [B, nmodes, T], trace flags
    [B, T], counters, cmax).
    """

    def __init__(self, nc=512, cmin=0.2, cmax=None, c_tol_rel=1e-6, f_accept=1.0, block=256):
        if nc < 3:
            raise ValueError(f"nc must be at least 3, got {nc}")
        if cmin <= 0:
            raise ValueError(f"cmin must be positive, got {cmin}")
        self.nc, self.cmin, self.cmax = int(nc), float(cmin), None if cmax is None else float(cmax)
        self.c_tol_rel, self.f_accept, self.block = float(c_tol_rel), float(f_accept), int(block)
        self._scan = self._ref = None
        self._key = None
        self._periods = None

    def close(self):
        for stage in (self._scan, self._ref):
            if stage is not None:
                stage.close()
        self._scan = self._ref = None
        self._key = self._periods = None

    def __call__(self, thickness, vp, vs, rho, periods, nmodes=5):
        from . import plugin
        if not isinstance(nmodes, (int, np.integer)) or nmodes < 1:
            raise ValueError(f"nmodes must be at least 1, got {nmodes}")
        d = _as_2d(thickness, "thickness")
        a = _as_2d(vp, "vp", d.shape[0])
        b = _as_2d(vs, "vs", d.shape[0])
        r = _as_2d(rho, "rho", d.shape[0])
        if not (d.shape == a.shape == b.shape == r.shape):
            raise ValueError(f"thickness/vp/vs/rho must all have the same shape, got {d.shape}, {a.shape}, "
                             f"{b.shape}, {r.shape}")
        B, L = d.shape
        if B < 1:
            raise ValueError("batch must contain at least one model")
        if L < 2:
            raise ValueError(f"need at least 2 layers (one plus the half-space), got L={L}")
        for name, arr in (("thickness", d), ("vp", a), ("vs", b), ("rho", r)):
            if not np.all(np.isfinite(arr)):
                raise ValueError(f"{name} must be finite everywhere")
        if np.any(d < 0):
            raise ValueError("thickness must be non-negative; the last entry is the half-space and its "
                             "thickness is ignored")
        for name, arr in (("vp", a), ("vs", b), ("rho", r)):
            if np.any(arr <= 0):
                raise ValueError(f"{name} must be positive; a zero or negative value is not a solid layer "
                                 f"(fluid layers are deliberately out of scope)")
        if np.any(a <= b):
            raise ValueError("vp must exceed vs in every layer; a P velocity at or below the S velocity is "
                             "not an elastic solid")
        per = np.ascontiguousarray(periods, dtype=np.float64)
        if per.ndim != 1 or per.size == 0:
            raise ValueError("periods must be a non-empty 1-D array")
        if not np.all(np.isfinite(per)):
            raise ValueError("periods must be finite (inf passes a > 0 test)")
        if not np.all(per > 0):
            raise ValueError("periods must be positive")
        ceiling = float(b[:, -1].max())
        cmax = self.cmax
        if cmax is None:
            cmax = ceiling
        elif cmax > ceiling:
            raise ValueError(f"cmax={cmax:g} is above the largest half-space Vs in the batch ({ceiling:g}); "
                             f"trapped Rayleigh modes do not exist there")
        if cmax <= self.cmin:
            raise ValueError(f"cmax ({cmax}) must exceed cmin ({self.cmin}); the scan range is empty")
        key = (B, L, per.size, self.nc, int(nmodes))
        if key != self._key:
            self.close()
            self._scan, self._ref = plugin.CoarseScan(B, L), plugin.Refine(B, L)
            for stage in (self._scan, self._ref):
                stage.upload_periods(per)
            self._scan.allocate(self.nc)
            self._ref.allocate(self.nc, int(nmodes))
            self._key = key
            self._periods = per.copy()
        elif not np.array_equal(self._periods, per):
            for stage in (self._scan, self._ref):
                stage.upload_periods(per)
            self._periods = per.copy()
        self._scan.upload_models(d, a, b, r)
        self._ref.upload_models(d, a, b, r)
        self._scan.run(self.cmin, cmax, self.block)
        self._ref.run(self._scan, self.cmin, cmax, self.c_tol_rel, self.f_accept, int(nmodes), self.block)
        return self._ref.download(), self._ref.flags(), self._ref.stats(), cmax

    def kernel_report(self):
        if self._scan is None:
            raise RuntimeError("call the solver first")
        return {"coarse_scan": self._scan.kernel_report(self.block), "refine": self._ref.kernel_report(self.block)}
