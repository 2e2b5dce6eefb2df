"""Cross-period mode-reliability checks on the GPU.

    r = check_mode_reliability(result)          # a DispersionBatch
    r = check_mode_reliability(velocity, periods, trace_flags=..., root_count=...)
    r.flags, r.assessed, r.passes_checks, r.summary()

The same conservative checks, flags and API as the reference's
``check_mode_reliability`` (python/modisp/reliability.py:49-145): ranks are
compared across sorted periods without editing the solution; a smooth wrong or
missing branch can pass.  Validation and the period plan (stable sort, distinct
periods, gaps, prediction ratios -- T entries, computed here with the
reference's own numpy arithmetic so every ratio is bit-identical) run on the
host; the B x K x T cell checks run in the engine's ``mode_reliability`` kernel
(``md200_mode_reliability``), one thread per (model, period).
"""
from __future__ import annotations

from dataclasses import dataclass
from enum import IntFlag

import numpy as np

from . import _native


class ModeReliabilityFlag(IntFlag):
    """Per-cell reliability flags (python/modisp/reliability.py:12-24)."""
    UNASSESSED = 1
    NUMERICAL_FAILURE = 2
    ROOT_COUNT_CHANGE = 4
    CLOSE_ROOT = 8
    RANK_AMBIGUOUS = 16
    STEP_JUMP = 32
    PREDICTION_MISMATCH = 64
    DUPLICATE_MISMATCH = 128
    NONFINITE = 256
    PERIOD_GAP = 512
    SEARCH_UNCERTAIN = 1024


@dataclass(frozen=True)
class ModeReliability:
    """Result of check_mode_reliability (python/modisp/reliability.py:27-46)."""
    flags: np.ndarray           # [B,K,T] uint16, original period order
    assessed: np.ndarray        # [B,K,T] bool: a finite, sufficiently sampled incoming edge
    previous_index: np.ndarray  # [T] original index of the previous distinct period, -1 first
    sorted_order: np.ndarray    # [T] stable period sort

    @property
    def suspect(self):
        return self.flags != 0

    @property
    def passes_checks(self):
        """Passed the observed checks; not a certificate of modal identity or completeness."""
        return self.assessed & ~self.suspect

    def summary(self):
        return dict(cells=int(self.flags.size), assessed=int(self.assessed.sum()),
                    passes_checks=int(self.passes_checks.sum()),
                    flags={f.name: int(np.count_nonzero(self.flags & int(f))) for f in ModeReliabilityFlag})


def _log_gap(a, b):
    """ln(b / a), a <= b, keeping adjacent representable periods distinct
    (python/modisp/reliability.py:7-9; the same numpy operations)."""
    return float(np.log1p((b - a) / a)) if b - a < a else float(np.log(b) - np.log(a))


def period_plan(periods, max_log_period_gap=.25):
    """The period walk of the checks (python/modisp/reliability.py:107-144) as a
    plan of T entries: (plan [T] md200_period_plan, order [T] int32, previous [T])."""
    p = np.asarray(periods, dtype=float)
    T = p.size
    order = np.argsort(p, kind="stable")
    plan = np.zeros(T, _native.PERIOD_PLAN)
    plan["prev"] = -1
    plan["older"] = -1
    previous = np.full(T, -1, dtype=np.int64)
    unique: list[int] = []
    for q, idx in enumerate(order):
        idx = int(idx)
        e = plan[idx]
        if not unique:
            e["kind"] = _native.PLAN_FIRST
        else:
            prev = unique[-1]
            e["prev"] = prev
            previous[idx] = prev
            if p[idx] == p[prev]:
                e["kind"] = _native.PLAN_DUPLICATE
                plan[prev]["dup_end"] = q + 1
                continue
            gap = _log_gap(p[prev], p[idx])
            kind = _native.PLAN_GAP if gap > max_log_period_gap else 0
            if len(unique) >= 2:
                older = unique[-2]
                den = _log_gap(p[older], p[prev])
                if den <= max_log_period_gap and gap <= max_log_period_gap:
                    kind |= _native.PLAN_PREDICT
                    e["older"] = older
                    e["ratio"] = gap / den
            e["kind"] = kind
        e["dup_begin"] = e["dup_end"] = q + 1
        unique.append(idx)
    return plan, order.astype(np.int32), previous


def check_mode_reliability(result, periods=None, *, trace_flags=None, root_count=None, close_root_rtol=None,
                           max_relative_step=.1, prediction_rtol=.05, max_log_period_gap=.25, device=0):
    """Check recovered ranks across sorted periods without editing the solution.

    Pass a DispersionBatch, or velocity [B,K,T] plus periods [T].  Thresholds are
    heuristics; duplicates are compared separately; large gaps and the first
    period are explicitly unassessed.  Output indexing follows the input order.
    Argument checks and messages follow python/modisp/reliability.py:49-90.
    """
    if hasattr(result, "phase_velocity"):
        if periods is not None or trace_flags is not None or root_count is not None:
            raise ValueError("periods/trace_flags/root_count are supplied by the result")
        periods, trace_flags, root_count = result.period, result.trace_flags, result.root_count
        if close_root_rtol is None:
            close_root_rtol = result.close_root_rtol
        velocity = result.phase_velocity
    else:
        velocity = result
    if close_root_rtol is None:
        close_root_rtol = .005
    if np.iscomplexobj(velocity) or np.iscomplexobj(periods):
        raise ValueError("velocities and periods must be real")
    v = np.asarray(velocity, dtype=float)
    p = np.asarray(periods, dtype=float)
    if (v.ndim != 3 or min(v.shape) < 1 or p.ndim != 1 or len(p) != v.shape[2] or not np.isfinite(p).all()
            or np.any(p <= 0)):
        raise ValueError("expected velocity [B,K,T] and finite positive periods [T]")
    if np.isinf(v).any() or np.any(v[np.isfinite(v)] <= 0):
        raise ValueError("velocities must be positive finite values or NaN")
    for name, x in (("close_root_rtol", close_root_rtol), ("max_relative_step", max_relative_step),
                    ("prediction_rtol", prediction_rtol), ("max_log_period_gap", max_log_period_gap)):
        if not np.isscalar(x) or np.iscomplexobj(x) or not np.isfinite(x) or x <= 0:
            raise ValueError(f"{name} must be finite and positive")
    B, K, T = v.shape
    tf = None
    if trace_flags is not None:
        tf = np.asarray(trace_flags)
        if tf.shape != (B, T) or tf.dtype.kind not in "iu" or np.any(tf < 0):
            raise ValueError("trace_flags must be nonnegative integer [B,T]")
        tf = tf.astype(np.uint32)  # every bit the checks read lies in the low 32
    counts = None
    if root_count is not None:
        counts = np.asarray(root_count)
        if counts.shape != (B, T) or counts.dtype.kind not in "iu":
            raise ValueError("root_count must be integer [B,T]")
        counts = counts.astype(np.int64)
    plan, order, previous = period_plan(p, max_log_period_gap)
    flags, assessed = _native.mode_reliability(v, plan, order, tf, counts, float(close_root_rtol),
                                               float(max_relative_step), float(prediction_rtol), device)
    return ModeReliability(flags, assessed, previous, order.astype(np.int64))
