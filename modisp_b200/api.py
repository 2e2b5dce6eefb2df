"""modisp's public API (`dispersion`, `dispersion_batch`, `Solver`) on the B200 engine.

Same call signatures, validation rules, result type and flag values as
python/modisp/__init__.py (file:line cited per item), so code written against
modisp runs unchanged.  The engine runs every trace on the GPU: there is no CPU
path here and a missing engine library or GPU raises BackendUnavailableError.
"""
from __future__ import annotations

import os
import threading
import time
from enum import IntEnum, IntFlag

import numpy as np

from . import _native
from ._native import BackendUnavailableError

__version__ = "0.5.0"

# Trace flag bits (python/modisp/__init__.py:15-32).
TRACE_UNRESOLVED_BRACKET = 1
TRACE_RELOCATED = 2
TRACE_SEARCH_UNCONVERGED = 4
TRACE_WORKSPACE_LIMIT = 8
TRACE_NEAR_CUTOFF = 16
TRACE_NONFINITE = 32
TRACE_REFINEMENT_FAILED = 64
TRACE_F_REJECTED = 128
TRACE_RANGE_TRUNCATED = 256
TRACE_SAMPLING_UNCERTAIN = 512
TRACE_ROOT_CONFLICT = 1024
TRACE_APPROXIMATE_SEARCH = 2048
TRACE_CLOSE_ROOT_RISK = 4096
TRACE_ADAPTIVE_FALLBACK = 8192
TRACE_LOVE_PHASE_FALLBACK = 16384
TRACE_FP64_REPAIR = 32768
TRACE_CONTINUATION_APPROXIMATE = 65536
TRACE_AUTO_RELAXED = 1 << 17
DEFAULT_ACCURACY = "auto"
_ACCURACY_CODE = {"high": 0, "balanced": 1, "fast": 2, "uniform": 3, "auto": 4}

# Search levels of this engine.
LEVEL_FP64_SCAN = 20
LEVEL_FP32_SCAN = 21
LEVEL_FP32_REPAIRED = 22
LEVEL_CONTINUATION = 23


class SolveStatus(IntEnum):
    """python/modisp/__init__.py:39-43"""
    VALID = 0
    NOT_FOUND = 1
    UNRESOLVED = 2
    REJECTED = 3


class GroupVelocityFlag(IntFlag):
    """python/modisp/__init__.py:46-52"""
    MISSING_ROOT = 1
    POLISH_FAILED = 2
    DERIVATIVE_UNSTABLE = 4
    ILL_CONDITIONED = 8
    CLOSE_ROOT = 16
    NONFINITE = 32


class PredictionFlag(IntFlag):
    """python/modisp/__init__.py:55-68"""
    ANCHOR = 1
    ACCEPTED = 2
    FALLBACK = 4
    BYPASSED = 8
    AUDIT = 16
    AUDIT_FAILED = 32
    SOURCE_SEARCH_UNCERTAIN = 64
    ROOT_COUNT_UNSAFE = 128
    ANCHOR_UNSAFE = 256
    WINDOW_UNSAFE = 512
    BRACKET_FAILED = 1024
    CORRECTION_FAILED = 2048
    REVIEW = 4096


class DispersionBatch:
    """Result of one solve (python/modisp/__init__.py:71-139): the same fields and masks."""

    def __init__(self, velocity, periods, nmodes, wave, flags, levels, counts, bounds, backend, reason,
                 accuracy=None, close_root_rtol=.005, search_strategy=None, sampling_rtol=None,
                 secular=None, refinement=None, love_strategy=None, group_velocity=None,
                 group_velocity_flags=None, prediction_flags=None, group_rtol=None,
                 frequency_strategy="independent", frequency_strategy_used="independent",
                 frequency_strategy_reason="independent frequency search requested", anchor_stride=4,
                 continuity_flags=None):
        self.phase_velocity = velocity
        self.precision = velocity.dtype.name
        self.refinement = refinement
        self.love_strategy = love_strategy
        self.secular = secular
        self.period = np.array(periods, copy=True)
        self.mode = np.arange(nmodes)
        self.wave = wave
        self.accuracy = accuracy
        self.search_strategy = search_strategy
        self.sampling_rtol = sampling_rtol
        self.close_root_rtol = float(close_root_rtol)
        self.group_velocity = group_velocity
        self.group_velocity_flags = group_velocity_flags
        self.group_velocity_mask = (None if group_velocity is None
                                    else np.isfinite(group_velocity) & (group_velocity_flags == 0))
        self.group_velocity_valid = self.group_velocity_mask
        self.prediction_flags = prediction_flags
        self.continuity_flags = continuity_flags
        self.group_rtol = group_rtol
        self.frequency_strategy = frequency_strategy
        self.frequency_strategy_used = frequency_strategy_used
        self.frequency_strategy_reason = frequency_strategy_reason
        self.anchor_stride = int(anchor_stride)
        self.approximate_search = (flags & (TRACE_APPROXIMATE_SEARCH | TRACE_CONTINUATION_APPROXIMATE)) != 0
        self.mode_index_uncertain = self.approximate_search.copy()
        self.close_root_mask = np.zeros(velocity.shape, dtype=bool)
        if nmodes > 1:
            gaps = np.diff(velocity, axis=1)
            close = np.isfinite(gaps) & (gaps <= self.close_root_rtol * velocity[:, 1:, :])
            self.close_root_mask[:, :-1, :] |= close
            self.close_root_mask[:, 1:, :] |= close
        self.close_root_risk = ((flags & TRACE_CLOSE_ROOT_RISK) != 0) | np.any(self.close_root_mask, axis=1)
        self.potentially_ambiguous = self.mode_index_uncertain | self.close_root_risk
        self.mode_mask = np.isfinite(velocity)
        self.trace_flags = flags
        self.numerical_flags = flags & np.uint32(0xFFFFFFFF ^ (TRACE_RANGE_TRUNCATED | TRACE_AUTO_RELAXED))
        self.search_level = levels
        self.root_count = counts
        self.search_bounds = np.array(bounds, copy=True)
        self.backend_used = backend
        self.backend_reason = reason
        self.status = np.where(self.mode_mask, SolveStatus.VALID,
                               np.where((flags[:, None, :] & (TRACE_SEARCH_UNCONVERGED | TRACE_UNRESOLVED_BRACKET)) != 0,
                                        SolveStatus.UNRESOLVED, SolveStatus.NOT_FOUND)).astype(np.uint8)
        rejected = (np.isnan(velocity) & ((flags[:, None, :] & TRACE_F_REJECTED) != 0)
                    & (np.arange(nmodes)[None, :, None] < counts[:, None, :]))
        self.status[rejected] = SolveStatus.REJECTED
        self.mode_convention = "ascending roots in the reported search interval"

    @property
    def auto_relaxed(self):
        """Traces whose accepted search used a wider automatic sampling tolerance
        (python/modisp/__init__.py:129-132); None unless accuracy is "auto"."""
        return (self.trace_flags & TRACE_AUTO_RELAXED) != 0 if self.accuracy == "auto" else None

    def check_modes(self, **options):
        """Cross-period mode-reliability checks of this result on the GPU
        (python/modisp/__init__.py:126-127); see modisp_b200.reliability."""
        from .reliability import check_mode_reliability
        return check_mode_reliability(self, **options)

    @property
    def n_models(self):
        return self.phase_velocity.shape[0]

    @property
    def n_modes(self):
        return self.phase_velocity.shape[1]

    def __len__(self):
        return self.n_models

    def __repr__(self):
        return (f"<DispersionBatch {self.wave} backend={self.backend_used} B={self.n_models} "
                f"nmodes={self.n_modes} T={self.period.size}>")


def _models(thickness, vp, vs, rho):
    """Validation of python/modisp/__init__.py:142-157 (same rules and messages)."""
    arrays = []
    for name, value in zip(("thickness", "vp", "vs", "rho"), (thickness, vp, vs, rho)):
        if np.iscomplexobj(value):
            raise ValueError(f"{name} must be real")
        a = np.ascontiguousarray(value, dtype=np.float64)
        if a.ndim == 1:
            a = a[None, :]
        if a.ndim != 2 or not a.size or not np.isfinite(a).all():
            raise ValueError(f"{name} must be a finite nonempty [B,L] or [L] array")
        arrays.append(a)
    h, a, b, r = arrays
    if any(v.shape != h.shape for v in arrays):
        raise ValueError("model array shapes must agree")
    if h.shape[1] > 256:
        raise ValueError("at most 256 layers are supported")
    if np.any(h < 0) or np.any(a <= 0) or np.any(r <= 0) or np.any(b < 0):
        raise ValueError("thickness/vs must be non-negative and vp/rho positive")
    if np.any(b[:, -1] <= 0) or np.any(b[:, 1:] == 0):
        raise ValueError("only a single first water layer may have vs=0; the half-space must be solid")
    solid = b > 0
    if np.any(a[solid] / b[solid] <= np.sqrt(4. / 3.)):
        raise ValueError("solid vp/vs must exceed sqrt(4/3) for positive bulk modulus")
    return arrays


def _workspace_per_model(L, T, nmodes):
    """Device bytes the engine reserves per model of capacity."""
    K = nmodes + 2
    KB = K + 16
    per_trace = KB * 5 * 8 + 8 * 4 * 8 + KB * 4 + 8 * 4 + nmodes * (8 * 4 + 4 * 2 + 16) + 64
    Ls = (L + 3) & ~3
    return T * per_trace + 9 * Ls * 12 + (129 + 2 * L) * 32 + (6 * L + 32) * 8 + 96 + 4 * L * 8


class Solver:
    """Reusable dispersion solver on the B200 engine (python/modisp/__init__.py:160-564).

    Accepts the reference's keyword arguments.  backend may be "auto", "cuda" or
    "b200" (all select the engine).  precision is "float64" (FP64 scan and
    refinement), "mixed" (FP32 scan, FP64 refinement, float64 results) or
    "float32" (the mixed engine with float32 results, as modisp returns them).
    Engine tuning: scan_density (scan points per phase unit), log_points,
    warps_per_block, blocks_per_sm; None keeps the engine defaults (or the
    autotuner's choice, see modisp_b200.autotune).
    """

    def __init__(self, nc=512, cmin=None, cmax=None, c_tol_rel=None, f_accept=1., block=256,
                 search_strategy="shape_adaptive", workspace_bytes=None, chunk_size=None, *,
                 backend="auto", device=0, threads=None, profile=False, accuracy=None,
                 adaptive_period_threshold=None, close_root_rtol=.005, sampling_rtol=None, secular=None,
                 refinement=None, love_strategy="phase", precision="float64", group_velocity=False,
                 group_rtol=.001, frequency_strategy="independent", anchor_stride=4,
                 continuity_check=True, scan_density=None, log_points=None, warps_per_block=None,
                 blocks_per_sm=None):
        if backend not in ("auto", "cuda", "b200"):
            if backend == "cpu":
                raise ValueError("modisp_b200 runs on the GPU only; use modisp's own CPU backend for backend='cpu'")
            raise ValueError("backend must be auto, cuda or b200")
        if search_strategy not in ("shape_adaptive", "qe_adaptive", "uniform"):
            raise ValueError("invalid search_strategy")
        if not isinstance(continuity_check, (bool, np.bool_)):
            raise ValueError("continuity_check must be boolean")
        if not isinstance(group_velocity, (bool, np.bool_)):
            raise ValueError("group_velocity must be boolean")
        if (not np.isscalar(group_rtol) or isinstance(group_rtol, (str, bytes, bool, np.bool_))
                or np.iscomplexobj(group_rtol) or not np.isfinite(group_rtol) or not 0 < group_rtol < 1):
            raise ValueError("group_rtol must be finite and between 0 and 1")
        if frequency_strategy not in ("independent", "anchor_continuation"):
            raise ValueError("frequency_strategy must be independent or anchor_continuation")
        if (not isinstance(anchor_stride, (int, np.integer)) or isinstance(anchor_stride, (bool, np.bool_))
                or anchor_stride < 2):
            raise ValueError("anchor_stride must be an integer of at least 2")
        uniform = search_strategy == "uniform"  # the legacy path (python/modisp/__init__.py:194-217)
        if uniform and (group_velocity or frequency_strategy != "independent"):
            raise NotImplementedError("group velocity and frequency continuation require an adaptive solver")
        if not isinstance(precision, str) or precision not in ("float64", "float32", "mixed"):
            raise ValueError("precision must be float64, mixed or float32")
        if uniform and precision != "float64":
            raise ValueError("precision='float32' requires an adaptive CUDA solver")
        if secular not in (None, "dunkin", "fast"):
            raise ValueError("secular must be None, 'dunkin' or 'fast'")
        if refinement is None:
            refinement = "legacy" if uniform else "brent"
        if refinement not in ("legacy", "brent", "chandrupatla"):
            raise ValueError("refinement must be legacy, brent or chandrupatla")
        if love_strategy not in ("phase", "scan"):
            raise ValueError("love_strategy must be phase or scan")
        if uniform and refinement != "legacy":
            raise NotImplementedError("uniform supports only legacy refinement")
        if uniform and secular == "fast":
            raise NotImplementedError("secular='fast' is not available on the legacy uniform CUDA path")
        if accuracy is None or (accuracy == "auto" and uniform):
            accuracy = "uniform" if uniform else DEFAULT_ACCURACY
        elif accuracy not in ("auto", "high", "balanced", "fast"):
            raise ValueError("accuracy must be auto, high, balanced or fast")
        elif uniform:
            raise ValueError("accuracy applies only to adaptive strategies; uniform is the legacy fixed path")
        if adaptive_period_threshold is not None:
            if accuracy in ("high", "uniform"):
                raise ValueError("adaptive_period_threshold applies only to auto/balanced/fast")
            if not np.isfinite(adaptive_period_threshold) or adaptive_period_threshold <= 0:
                raise ValueError("adaptive_period_threshold must be finite and positive")
        if (not np.isscalar(close_root_rtol) or np.iscomplexobj(close_root_rtol)
                or not np.isfinite(close_root_rtol) or not 0 < close_root_rtol < 1):
            raise ValueError("close_root_rtol must be finite and between 0 and 1")
        if sampling_rtol is not None and search_strategy != "shape_adaptive":
            raise ValueError("sampling_rtol applies only to shape_adaptive")
        if sampling_rtol is None:
            sampling_rtol = {"auto": 1e-2, "high": 1e-3, "balanced": 1e-2, "fast": 5e-2, "uniform": 1e-3}[accuracy]
        if (not np.isscalar(sampling_rtol) or np.iscomplexobj(sampling_rtol) or not np.isfinite(sampling_rtol)
                or not 0 < sampling_rtol <= 1):
            raise ValueError("sampling_rtol must be finite and between 0 and 1")
        if c_tol_rel is None:
            c_tol_rel = {"auto": 1e-5, "high": 1e-6, "balanced": 1e-5, "fast": 1e-4, "uniform": 1e-6}[accuracy]
        for name, v in (("cmin", cmin), ("cmax", cmax)):
            if v is not None and (not np.isfinite(v) or v <= 0):
                raise ValueError(f"{name} must be finite and positive")
        if cmin is not None and cmax is not None and cmax <= cmin:
            raise ValueError("cmax must exceed cmin")
        if not np.isfinite(c_tol_rel) or c_tol_rel <= 0:
            raise ValueError("c_tol_rel must be positive")
        if not np.isfinite(f_accept) or f_accept < 0:
            raise ValueError("f_accept must be non-negative")
        if nc < 3:
            raise ValueError("nc must be at least 3")
        if workspace_bytes is not None and (not isinstance(workspace_bytes, (int, np.integer)) or workspace_bytes < 1):
            raise ValueError("workspace_bytes must be a positive integer")
        if chunk_size is not None and (not isinstance(chunk_size, (int, np.integer)) or chunk_size < 1):
            raise ValueError("chunk_size must be positive")
        if not isinstance(device, (int, np.integer)) or device < 0:
            raise ValueError("device must be a non-negative integer")
        if not isinstance(profile, (bool, np.bool_)):
            raise ValueError("profile must be boolean")
        self.nc, self.cmin, self.cmax = int(nc), cmin, cmax
        self.c_tol_rel, self.f_accept, self.block = float(c_tol_rel), float(f_accept), int(block)
        self.search_strategy, self.workspace_bytes, self.chunk_size = search_strategy, workspace_bytes, chunk_size
        self.backend, self.device, self.threads = backend, int(device), threads
        self.profile, self.accuracy, self.adaptive_period_threshold = bool(profile), accuracy, adaptive_period_threshold
        self.close_root_rtol, self.sampling_rtol, self.secular = float(close_root_rtol), float(sampling_rtol), secular
        self.refinement, self.love_strategy, self.precision = refinement, love_strategy, precision
        self.group_velocity, self.group_rtol = bool(group_velocity), float(group_rtol)
        self.frequency_strategy, self.anchor_stride = frequency_strategy, int(anchor_stride)
        self.continuity_check = bool(continuity_check)
        self.tuning = dict(scan_density=scan_density, log_points=log_points,
                           warps_per_block=warps_per_block, blocks_per_sm=blocks_per_sm)
        self._engine = None
        self._engine_key = None
        self._legacy = None
        self._calls = 0
        self._last_stats = None
        self.last_result = None
        self._lock = threading.RLock()

    # -- backend -----------------------------------------------------------
    def _select(self):
        from . import plugin
        if not plugin.available(self.device):
            raise BackendUnavailableError(f"B200 engine: CUDA device {self.device} is unavailable")
        plugin.set_device(self.device)
        return "cuda", "B200 engine and sm_100 device available"

    def _capacity(self, B, L, T, nmodes):
        per_model = _workspace_per_model(L, T, nmodes)
        if self.workspace_bytes is not None:
            limit = max(1, int(self.workspace_bytes) // per_model)
            if self.workspace_bytes < per_model:
                raise MemoryError("workspace_bytes is too small for one model; increase the budget")
        else:
            free, _ = _native.memory_info()
            limit = max(1, int(0.4 * free) // per_model)
        return max(1, min(B, limit, self.chunk_size or B))

    def _engine_for(self, capacity, L, T, nmodes, continuation=False):
        from . import plugin
        key = (self.device, L, T, int(nmodes), self.accuracy, self.close_root_rtol, self.precision,
               self.group_velocity, bool(continuation), self.anchor_stride, self.continuity_check,
               tuple(sorted(self.tuning.items())))
        if self._engine is not None and self._engine_key[0] == key and self._engine_key[1] >= capacity:
            return self._engine, False
        self.close()
        t = {k: (v or 0) for k, v in self.tuning.items()}
        self._engine = plugin.QeSolver(
            capacity, L, T, int(nmodes), _ACCURACY_CODE[self.accuracy], 0., self.close_root_rtol, True,
            self.sampling_rtol, 1 if self.secular == "fast" else 0,
            {"legacy": 0, "brent": 1, "chandrupatla": 2}[self.refinement], int(self.love_strategy == "phase"),
            self.precision != "float64", self.group_velocity, self.group_rtol,
            bool(continuation), self.anchor_stride,
            scan_density=float(t["scan_density"]), log_points=int(t["log_points"]),
            warps_per_block=int(t["warps_per_block"]), blocks_per_sm=int(t["blocks_per_sm"]),
            continuity_check=self.continuity_check, device=self.device)
        self._engine_key = (key, capacity)
        return self._engine, True

    # -- solve -------------------------------------------------------------
    def __call__(self, thickness, vp, vs, rho, periods, nmodes=5, wave="rayleigh", names=None):
        if not self._lock.acquire(blocking=False):
            raise RuntimeError("a Solver instance cannot be used concurrently; create one instance per caller")
        try:
            return self._solve(thickness, vp, vs, rho, periods, nmodes, wave)
        finally:
            self._lock.release()

    def _solve(self, thickness, vp, vs, rho, periods, nmodes=5, wave="rayleigh"):
        started = time.perf_counter()
        if wave not in ("rayleigh", "love"):
            raise ValueError("wave must be rayleigh or love")
        if not isinstance(nmodes, (int, np.integer)) or not 1 <= nmodes <= 256:
            raise ValueError("nmodes must be 1..256")
        h, a, b, r = _models(thickness, vp, vs, rho)
        B, L = h.shape
        if np.iscomplexobj(periods):
            raise ValueError("periods must be real")
        per = np.ascontiguousarray(periods, dtype=np.float64)
        if per.ndim != 1 or not per.size or not np.isfinite(per).all() or np.any(per <= 0):
            raise ValueError("periods must be a finite positive 1-D array")
        if self.precision != "float64":
            fp32 = np.finfo(np.float32)
            max_value, zero_cutoff = float(fp32.max), .5 * float(fp32.smallest_subnormal)
            for name, values in zip(("thickness", "vp", "vs", "rho"), (h, a, b, r)):
                if values.max() > max_value or np.any((values > 0.) & (values <= zero_cutoff)):
                    raise ValueError(f"{name} contains values outside the float32 range")
            if per.max() > max_value or per.min() < 2. * np.pi / max_value:
                raise ValueError("periods or their angular frequencies are outside the float32 range")
        backend, reason = self._select()
        if self.search_strategy == "uniform":
            return self._solve_uniform(h, a, b, r, per, nmodes, wave, backend, reason, started)
        input_periods = per
        inverse = None
        # frequency strategy (python/modisp/__init__.py:318-340): continuation runs on
        # sorted unique periods for the approximate presets
        continuation = False
        frequency_reason = "independent frequency search requested"
        if self.frequency_strategy == "anchor_continuation":
            unique = np.unique(per)
            if self.accuracy == "high":
                frequency_reason = "high accuracy retains independent search"
            elif unique.size < 8:
                frequency_reason = "fewer than 8 unique periods; using independent search"
            elif not np.any(np.log(unique[2:]) - np.log(unique[:-2]) <= .25):
                frequency_reason = ("period grid has no interior target within the anchor log-gap limit; "
                                    "using independent search")
            else:
                continuation = True
                frequency_reason = "CUDA anchor continuation on sorted unique periods"
        if continuation or (per.size > 1 and not np.all(per[1:] > per[:-1]) and not np.all(per[1:] < per[:-1])):
            per, inverse = np.unique(per, return_inverse=True)  # python/modisp/__init__.py:314-341
        bounds_in = np.zeros((B, 2))
        bounds_in[:, 0] = self.cmin if self.cmin is not None else 0.
        bounds_in[:, 1] = self.cmax if self.cmax is not None else np.inf
        capacity = self._capacity(B, L, per.size, nmodes)
        engine, allocated = self._engine_for(capacity, L, per.size, nmodes, continuation)
        dtype = np.float32 if self.precision == "float32" else np.float64
        velocity = np.empty((B, nmodes, per.size), dtype=dtype)
        flags = np.empty((B, per.size), np.uint32)
        levels = np.empty((B, per.size), np.int32)
        counts = np.empty((B, per.size), np.int32)
        bounds = np.empty((B, 2))
        group = np.empty((B, nmodes, per.size)) if self.group_velocity else None
        gflags = np.empty((B, nmodes, per.size), np.uint32) if self.group_velocity else None
        # the continuity screen runs in the FP32-scan engine (continuity_check)
        screened = self.precision != "float64" and self.continuity_check
        cflags = np.empty((B, per.size), np.uint8) if screened else None
        # PredictionFlag words: BYPASSED (8) unless continuation assigns them
        pflags = (np.full((B, per.size), 8, np.uint32) if self.frequency_strategy == "anchor_continuation"
                  else None)
        stats = {}
        chunks = 0
        wave_code = int(wave == "love")
        for start in range(0, B, capacity):
            end = min(B, start + capacity)
            out = engine._engine.run(h[start:end], a[start:end], b[start:end], r[start:end], per,
                                     bounds_in[start:end], self.c_tol_rel, self.f_accept, wave_code,
                                     group=self.group_velocity, continuity=screened, prediction=continuation)
            velocity[start:end] = out["velocity"]
            flags[start:end] = out["flags"]
            levels[start:end] = out["levels"]
            counts[start:end] = out["counts"]
            bounds[start:end] = out["bounds"]
            if self.group_velocity:
                group[start:end] = out["group_velocity"]
                gflags[start:end] = out["group_velocity_flags"]
            if screened:
                cflags[start:end] = out["continuity_flags"]
            if continuation:
                pflags[start:end] = out["prediction_flags"]
            for k, v in out["stats"].items():
                stats[k] = stats.get(k, 0) + int(v)
            chunks += 1
        if not np.isfinite(bounds).all() or np.any(bounds[:, 0] <= 0):
            raise ValueError("automatic search range could not be constructed")
        if inverse is not None:
            velocity, flags, levels, counts = (x.take(inverse, axis=-1) for x in (velocity, flags, levels, counts))
            if cflags is not None:
                cflags = cflags.take(inverse, axis=-1)
            if pflags is not None:
                pflags = pflags.take(inverse, axis=-1)
            if group is not None:
                group, gflags = group.take(inverse, axis=-1), gflags.take(inverse, axis=-1)
        if self.cmin is not None or self.cmax is not None:
            flags |= TRACE_RANGE_TRUNCATED
        counts[(flags & TRACE_SEARCH_UNCONVERGED) != 0] = -1
        secular = self.secular or "fast"
        stats.update(backend=backend, precision=self.precision, strategy="b200_scan",
                     requested_strategy=self.search_strategy, accuracy=self.accuracy, secular=secular,
                     secular_kernel="sh" if wave == "love" else "dunkin",
                     refinement="brent", love_strategy=self.love_strategy if wave == "love" else None,
                     close_root_rtol=self.close_root_rtol, refinement_tolerance=self.c_tol_rel, chunks=chunks,
                     capacity_models=int(capacity), engine_allocations=int(allocated),
                     group_velocity=self.group_velocity, group_rtol=self.group_rtol,
                     frequency_strategy=self.frequency_strategy,
                     frequency_strategy_used="anchor_continuation" if continuation else "independent",
                     frequency_strategy_reason=frequency_reason,
                     periods_requested=int(input_periods.size), periods_computed=int(per.size),
                     close_root_risk_traces=int(np.count_nonzero(flags & TRACE_CLOSE_ROOT_RISK)),
                     threads=0)
        if self.profile:
            stats["timings_s"] = {"solver_total": time.perf_counter() - started}
        self._last_stats = stats
        self._calls += 1
        result = DispersionBatch(
            velocity, input_periods, nmodes, wave, flags, levels, counts, bounds, backend, reason,
            accuracy=self.accuracy, close_root_rtol=self.close_root_rtol, search_strategy=self.search_strategy,
            sampling_rtol=self.sampling_rtol, secular=secular, refinement=self.refinement,
            love_strategy=self.love_strategy if wave == "love" else None, group_velocity=group,
            group_velocity_flags=gflags, prediction_flags=pflags,
            group_rtol=self.group_rtol if self.group_velocity else None,
            frequency_strategy=self.frequency_strategy,
            frequency_strategy_used="anchor_continuation" if continuation else "independent",
            frequency_strategy_reason=frequency_reason, anchor_stride=self.anchor_stride, continuity_flags=cflags)
        self.last_result = result
        return result

    def _solve_uniform(self, h, a, b, r, per, nmodes, wave, backend, reason, started):
        """The legacy uniform path as the reference's Solver wraps it
        (python/modisp/__init__.py:302-311): solid Rayleigh only, cmin 0.2 unless
        given, every trace flagged TRACE_RANGE_TRUNCATED, search level -2."""
        from .legacy import UniformSolver
        B, L = h.shape
        if wave != "rayleigh" or np.any(b == 0) or L < 2:
            raise NotImplementedError("uniform is the legacy CUDA solid-Rayleigh option; use qe_adaptive for this "
                                      "combination")
        cmin = .2 if self.cmin is None else self.cmin
        if self._legacy is None:
            self._legacy = UniformSolver(self.nc, cmin, self.cmax, self.c_tol_rel, self.f_accept, self.block)
        velocity, flags, legacy_stats, _ = self._legacy(h, a, b, r, per, nmodes)
        vs_hs = b[:, -1]
        bounds = np.empty((B, 2))
        bounds[:, 0] = cmin
        bounds[:, 1] = np.fmin(vs_hs if self.cmax is None else self.cmax, np.nextafter(vs_hs, 0.))
        flags = flags | TRACE_RANGE_TRUNCATED
        levels = np.full((B, per.size), -2, np.int32)
        counts = np.sum(np.isfinite(velocity), axis=1, dtype=np.int32)
        result = DispersionBatch(velocity, per, nmodes, wave, flags, levels, counts, bounds, backend, reason,
                                 accuracy="uniform", close_root_rtol=self.close_root_rtol, search_strategy="uniform",
                                 secular="dunkin", refinement="legacy")
        stats = dict(legacy_stats)
        stats.update(backend=backend, accuracy="uniform", precision=self.precision,
                     close_root_rtol=self.close_root_rtol, secular="dunkin", secular_kernel="dunkin",
                     refinement="legacy", love_strategy=None, group_velocity=False, group_rtol=self.group_rtol,
                     frequency_strategy="independent", frequency_strategy_used="independent",
                     anchor_stride=self.anchor_stride)
        if self.profile:
            stats["timings_s"] = {"solver_total": time.perf_counter() - started}
        self._last_stats = stats
        self._calls += 1
        self.last_result = result
        return result

    @property
    def calls(self):
        return self._calls

    def stats(self):
        if self._last_stats is None:
            raise RuntimeError("call the solver first")
        return dict(self._last_stats)

    def kernel_report(self):
        from . import plugin
        if self.search_strategy == "uniform" and self._legacy is not None:
            return {"backend": "cuda", "precision": "float32 scan / float64 refinement", "accuracy": "uniform",
                    "secular": "dunkin", "secular_kernel": "dunkin", "refinement": "legacy", "love_strategy": None,
                    "group_velocity": False, "frequency_strategy": "independent",
                    "frequency_strategy_used": "independent", "legacy": self._legacy.kernel_report()}
        L = self._engine.layers if self._engine is not None else 21
        report = plugin.qe_kernel_report(L, int(self.accuracy != "high"), True, self.precision != "float64")
        report.update(backend="cuda", precision=self.precision, accuracy=self.accuracy,
                      refinement=self.refinement, group_velocity=self.group_velocity)
        return report

    def close(self):
        with self._lock:
            if self._engine is not None:
                self._engine.close()
            self._engine = None
            self._engine_key = None
            if self._legacy is not None:
                self._legacy.close()
            self._legacy = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


_DEFAULT = None


def release():
    global _DEFAULT
    if _DEFAULT is not None:
        _DEFAULT.close()
        _DEFAULT = None


def dispersion_batch(thickness, vp, vs, rho, periods, nmodes=5, wave="rayleigh", solver=None, names=None,
                     search_strategy=None, accuracy=None, **options):
    """python/modisp/__init__.py:572-588"""
    global _DEFAULT
    if solver is not None:
        if options or (search_strategy is not None and search_strategy != solver.search_strategy) or \
                (accuracy is not None and accuracy != solver.accuracy):
            raise ValueError("options conflict with the supplied Solver")
        return solver(thickness, vp, vs, rho, periods, nmodes, wave, names)
    if options or accuracy is not None:
        with Solver(search_strategy="shape_adaptive" if search_strategy is None else search_strategy,
                    accuracy=accuracy, **options) as s:
            return s(thickness, vp, vs, rho, periods, nmodes, wave, names)
    strategy = "shape_adaptive" if search_strategy is None else search_strategy
    if _DEFAULT is None or _DEFAULT.search_strategy != strategy:
        release()
        _DEFAULT = Solver(search_strategy=strategy)
    return _DEFAULT(thickness, vp, vs, rho, periods, nmodes, wave, names)


def dispersion(model, periods, nmodes=5, wave="rayleigh", **options):
    """python/modisp/__init__.py:591-597: a model object, an [L, 4] array (h, vp, vs, rho) or a batch dict."""
    if isinstance(model, dict):
        batch = {k: model[k] for k in ("thickness", "vp", "vs", "rho")}
    elif all(hasattr(model, k) for k in ("thickness", "vp", "vs", "rho")):
        batch = {k: np.asarray(getattr(model, k)) for k in ("thickness", "vp", "vs", "rho")}
    else:
        arr = np.asarray(model)
        if arr.ndim != 2 or arr.shape[1] != 4:
            raise ValueError("model must be LayeredModel, an array with columns h/vp/vs/rho, or a batch dict")
        batch = dict(zip(("thickness", "vp", "vs", "rho"), arr.T))
    return dispersion_batch(**batch, periods=periods, nmodes=nmodes, wave=wave, **options)


def device_name():
    return _native.device_name(0)
