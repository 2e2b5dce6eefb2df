"""Oracle for the cross-period mode-reliability checks.

TEST INFRASTRUCTURE ONLY: imported by ``tests/`` and by the reference leg of
``bench.py`` to check (or time against) the engine's ``mode_reliability``
kernel; the product package never imports it.

A numpy restatement of the reference's conservative cross-period checks
(``python/modisp/reliability.py:49-145``), period by period, vectorised over
models and ranks and looping where the reference loops, so that its CPU time
stands for the reference's.  Pinned against fixtures that the reference module
itself produced (``tests/golden/reliability_*.npz``, made by
``tests/golden/make_golden.py``).
"""
from __future__ import annotations

import numpy as np

# Flag bits of ModeReliabilityFlag (python/modisp/reliability.py:12-24).
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

# Trace-flag bits that make a trace a numerical failure, and those that make its
# search uncertain (python/modisp/reliability.py:94-96).
FAILURE_TRACE_BITS = 1 | 4 | 8 | 32 | 64 | 128 | 512 | 1024
UNCERTAIN_TRACE_BITS = 2048 | 4096


def log_gap(a: float, b: float) -> float:
    """ln(b / a) for a <= b, through log1p when the gap is small so that adjacent
    representable periods stay distinct (python/modisp/reliability.py:7-9)."""
    return float(np.log1p((b - a) / a)) if b - a < a else float(np.log(b) - np.log(a))


def check(velocity, periods, trace_flags=None, root_count=None, close_root_rtol=.005, max_relative_step=.1,
          prediction_rtol=.05, max_log_period_gap=.25):
    """(flags uint16 [B,K,T], assessed bool [B,K,T], previous int64 [T], order int64 [T]).

    Vectorised over models and ranks as the reference is, looping over periods
    and (for the nearest-rank test) over models where it loops, so that its CPU
    time stands for the reference's.  Inputs are taken as already validated (the
    argument checks live in the product's Python layer and are tested there)."""
    v = np.asarray(velocity, dtype=float)
    p = np.asarray(periods, dtype=float)
    B, K, T = v.shape
    finite = np.isfinite(v)
    tf = np.zeros((B, T), np.uint32) if trace_flags is None else np.asarray(trace_flags)
    counts = finite.sum(axis=1) if root_count is None else np.asarray(root_count)
    flags = np.zeros(v.shape, np.uint16)
    assessed = np.zeros(v.shape, bool)
    previous = np.full(T, -1, np.int64)

    flags[~finite] |= NONFINITE
    failure = ((tf & FAILURE_TRACE_BITS) != 0) | (counts < 0)
    flags |= np.where(failure[:, None, :], NUMERICAL_FAILURE, 0).astype(np.uint16)
    flags |= np.where(((tf & UNCERTAIN_TRACE_BITS) != 0)[:, None, :], SEARCH_UNCERTAIN, 0).astype(np.uint16)
    # adjacent ranks: close pairs and order violations (:98-105)
    if K > 1:
        gap = v[:, 1:, :] - v[:, :-1, :]
        ok = np.isfinite(gap)
        close = ok & (gap <= close_root_rtol * v[:, 1:, :])
        bad = ok & (gap <= 0)
        for sl in (np.s_[:, :-1, :], np.s_[:, 1:, :]):
            flags[sl] |= np.where(close, CLOSE_ROOT, 0).astype(np.uint16)
            flags[sl] |= np.where(bad, RANK_AMBIGUOUS, 0).astype(np.uint16)

    # periods in stable sorted order (:107-144)
    order = np.argsort(p, kind="stable")
    unique: list[int] = []
    for idx in order:
        idx = int(idx)
        if not unique:
            flags[:, :, idx] |= UNASSESSED
            unique.append(idx)
            continue
        prev = unique[-1]
        previous[idx] = prev
        a, b = v[:, :, prev], v[:, :, idx]
        both = finite[:, :, prev] & finite[:, :, idx]
        fail2 = failure[:, prev, None] | failure[:, idx, None]
        changed = (counts[:, prev] != counts[:, idx]) | np.any(finite[:, :, prev] != finite[:, :, idx], axis=1)
        flags[:, :, idx] |= np.where(changed[:, None], ROOT_COUNT_CHANGE, 0).astype(np.uint16)
        if p[idx] == p[prev]:
            with np.errstate(invalid="ignore"):
                mismatch = (finite[:, :, prev] != finite[:, :, idx]) | (both & (np.abs(a - b) > 1e-10 * np.fmax(a, b)))
            flags[:, :, idx] |= np.where(mismatch, DUPLICATE_MISMATCH, 0).astype(np.uint16)
            flags[:, :, prev] |= np.where(mismatch, DUPLICATE_MISMATCH, 0).astype(np.uint16)
            assessed[:, :, idx] = both & ~fail2
            continue
        lg = log_gap(p[prev], p[idx])
        if lg > max_log_period_gap:
            flags[:, :, idx] |= PERIOD_GAP
        else:
            assessed[:, :, idx] = both & ~fail2
        with np.errstate(invalid="ignore", divide="ignore"):
            step = np.where(both, np.abs(b - a) / np.fmax(a, b), 0.)
        flags[:, :, idx] |= np.where(both & (step > max_relative_step), STEP_JUMP, 0).astype(np.uint16)
        # nearest-rank agreement, never a remapping (:129-135)
        for m in range(B):
            ia = np.flatnonzero(finite[m, :, prev])
            ib = np.flatnonzero(finite[m, :, idx])
            if not len(ia) or not len(ib):
                continue
            cost = np.abs(a[m, ia][:, None] - b[m, ib][None, :])
            col = np.argmin(cost, axis=0)
            row = np.argmin(cost, axis=1)
            ambiguous = (ia[col] != ib) | (ib[row][col] != ib)
            flags[m, ib[ambiguous], idx] |= RANK_AMBIGUOUS
        if len(unique) >= 2:
            older = unique[-2]
            den = log_gap(p[older], p[prev])
            if den <= max_log_period_gap and lg <= max_log_period_gap:
                valid = both & finite[:, :, older]
                with np.errstate(invalid="ignore"):
                    predicted = a + (a - v[:, :, older]) * (lg / den)
                    mismatch = valid & (np.abs(b - predicted) > prediction_rtol * b)
                flags[:, :, idx] |= np.where(mismatch, PREDICTION_MISMATCH, 0).astype(np.uint16)
        unique.append(idx)
    return flags, assessed, previous, order.astype(np.int64)
