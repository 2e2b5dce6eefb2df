"""Ragged batches: every model with its own periods and its own mode count.

    res = dispersion_ragged(thickness, vp, vs, rho, periods=[p0, p1, ...], nmodes=[3, 7, ...])
    res.phase_velocity_of(b)          # [nmodes[b], len(periods[b])] of model b

modisp's public API shares one period array across the batch
(python/modisp/__init__.py:285-286); a batch whose models carry different period
sets or mode counts would have to be split into uniform sub-batches.  Here the
whole batch runs as one set of launches: the engine's trace list holds every
(model, period) pair in CSR order and each trace carries its model, period,
mode count and output position (``md200_run_ragged``).  Outputs are flat: the
[nmodes[b], T_b] block of model b (mode, period -- the reference's layout per
model) at ``out_offsets[b]``; trace flags, levels and counts in CSR order.
Trace semantics (masks, counts, flags, group velocity) are those of the uniform
engine; the same parity bar applies per model.
"""
from __future__ import annotations

import numpy as np

from . import _native
from .api import _models

WAVES = {"rayleigh": 0, "love": 1}


class RaggedDispersion:
    """Results of a ragged batch (CSR layout)."""

    def __init__(self, period_offsets, periods, modes, out_offsets, velocity, flags, levels, counts, group,
                 group_flags, wave, stats):
        self.period_offsets = period_offsets
        self.periods = periods
        self.modes = modes
        self.out_offsets = out_offsets
        self.phase_velocity = velocity
        self.trace_flags = flags
        self.search_level = levels
        self.root_count = counts
        self.group_velocity = group
        self.group_velocity_flags = group_flags
        self.wave = wave
        self.stats = stats

    @property
    def n_models(self) -> int:
        return self.modes.size

    @property
    def n_roots(self) -> int:
        return int(np.isfinite(self.phase_velocity).sum())

    def _block(self, flat, b):
        T = int(self.period_offsets[b + 1] - self.period_offsets[b])
        start = int(self.out_offsets[b])
        return flat[start:start + int(self.modes[b]) * T].reshape(int(self.modes[b]), T)

    def periods_of(self, b):
        return self.periods[self.period_offsets[b]:self.period_offsets[b + 1]]

    def phase_velocity_of(self, b):
        """[nmodes[b], T_b] phase velocities of model b (NaN where no root)."""
        return self._block(self.phase_velocity, b)

    def group_velocity_of(self, b):
        return None if self.group_velocity is None else self._block(self.group_velocity, b)

    def mode_mask_of(self, b):
        return np.isfinite(self.phase_velocity_of(b))

    def root_count_of(self, b):
        return self.root_count[self.period_offsets[b]:self.period_offsets[b + 1]]

    def trace_flags_of(self, b):
        return self.trace_flags[self.period_offsets[b]:self.period_offsets[b + 1]]

    def __repr__(self):
        return (f"<RaggedDispersion {self.wave} B={self.n_models} traces={self.periods.size} "
                f"roots={self.n_roots}>")


def _csr(periods, B):
    if isinstance(periods, tuple) and len(periods) == 2:
        offsets = np.ascontiguousarray(periods[0], dtype=np.int64)
        flat = np.ascontiguousarray(periods[1], dtype=np.float64)
    else:
        if len(periods) != B:
            raise ValueError("periods needs one array per model")
        parts = [np.atleast_1d(np.asarray(p, dtype=np.float64)) for p in periods]
        offsets = np.zeros(B + 1, dtype=np.int64)
        offsets[1:] = np.cumsum([p.size for p in parts])
        flat = np.concatenate(parts) if parts else np.zeros(0)
    if offsets.size != B + 1 or offsets[0] != 0 or np.any(np.diff(offsets) < 0) or offsets[-1] != flat.size:
        raise ValueError("period offsets must start at 0, be non-decreasing and end at the period count")
    if flat.size and (not np.isfinite(flat).all() or np.any(flat <= 0)):
        raise ValueError("periods must be finite and positive")
    return offsets, flat


def dispersion_ragged(thickness, vp, vs, rho, periods, nmodes=5, wave="rayleigh", precision="mixed",
                      group_velocity=True, c_tol_rel=1e-10, f_accept=1., device=0, chunk_models=65536,
                      frequency_strategy="independent", anchor_stride=4):
    """Solve a ragged batch.

    ``periods``: a list of per-model period arrays, or a CSR pair (offsets [B+1],
    flat periods).  ``nmodes``: one count for all models or one per model.
    ``precision``: "mixed" (FP32 scan, FP64 refinement) or "float64".  Models are
    padded [B, L] arrays as in ``dispersion_batch``; chunks of ``chunk_models``
    models share one engine.  ``frequency_strategy="anchor_continuation"`` solves
    every ``anchor_stride``-th period of a model (its periods ascending, at least
    8) by the full search and predicts, refines and audits the periods between
    them, falling back to the full FP64 search on any doubt.
    """
    if wave not in WAVES:
        raise ValueError("wave must be 'rayleigh' or 'love'")
    if precision not in ("mixed", "float64"):
        raise ValueError("precision must be 'mixed' or 'float64'")
    if not (0. < c_tol_rel < 1.):
        raise ValueError("c_tol_rel must lie in (0, 1)")
    if frequency_strategy not in ("independent", "anchor_continuation"):
        raise ValueError("frequency_strategy must be independent or anchor_continuation")
    if not isinstance(anchor_stride, (int, np.integer)) or anchor_stride < 2:
        raise ValueError("anchor_stride must be an integer of at least 2")
    h, a, b, r = _models(thickness, vp, vs, rho)
    B, L = h.shape
    offsets, flat = _csr(periods, B)
    modes = np.broadcast_to(np.asarray(nmodes, dtype=np.int64), (B,)).copy()
    if np.any(modes < 1) or np.any(modes > 256):
        raise ValueError("nmodes must lie in 1..256")
    counts = np.diff(offsets)
    T_max = max(1, int(counts.max(initial=1)))
    nm_max = int(modes.max(initial=1))
    cells = modes * counts
    out_offsets = np.zeros(B, dtype=np.int64)
    out_offsets[1:] = np.cumsum(cells)[:-1]
    total_cells = int(cells.sum())
    velocity = np.full(total_cells, np.nan)
    group = np.full(total_cells, np.nan) if group_velocity else None
    gflags = np.zeros(total_cells, np.uint32) if group_velocity else None
    tflags = np.zeros(flat.size, np.uint32)
    levels = np.zeros(flat.size, np.int32)
    rcounts = np.zeros(flat.size, np.int32)
    stats = {}
    o = _native.default_options()
    o.single_precision = 1 if precision == "mixed" else 0
    o.group_velocity = int(bool(group_velocity))
    o.continuation = int(frequency_strategy == "anchor_continuation")
    o.anchor_stride = int(anchor_stride)
    cap = int(min(B, chunk_models))
    engine = _native.Engine(device, cap, L, T_max, nm_max, o)
    try:
        for s in range(0, B, cap):
            e = min(B, s + cap)
            sub_off = (offsets[s:e + 1] - offsets[s]).astype(np.int32)
            if sub_off[-1] == 0:
                continue
            out = engine.run_ragged(h[s:e], a[s:e], b[s:e], r[s:e], sub_off, flat[offsets[s]:offsets[e]],
                                    modes[s:e].astype(np.int32), c_tol_rel, f_accept, WAVES[wave],
                                    group=group_velocity)
            c0, c1 = int(out_offsets[s]), int(out_offsets[s] + cells[s:e].sum())
            t0, t1 = int(offsets[s]), int(offsets[e])
            velocity[c0:c1] = out["velocity"]
            tflags[t0:t1], levels[t0:t1], rcounts[t0:t1] = out["flags"], out["levels"], out["counts"]
            if group_velocity:
                group[c0:c1], gflags[c0:c1] = out["group_velocity"], out["group_velocity_flags"]
            for k, v in out["stats"].items():
                stats[k] = stats.get(k, 0) + v
    finally:
        engine.close()
    return RaggedDispersion(offsets, flat, modes, out_offsets, velocity, tflags, levels, rcounts, group, gflags,
                            wave, stats)
