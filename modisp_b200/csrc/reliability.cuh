// reliability.cuh -- cross-period mode-reliability checks on the device.
//
// The checks of the reference's check_mode_reliability
// (python/modisp/reliability.py:49-145): per cell, flags for non-finite roots,
// numerical-failure and uncertain-search trace bits, close and misordered
// adjacent ranks; then, in stable sorted period order, root-count changes,
// duplicate-period mismatches, period gaps, relative steps, nearest-rank
// ambiguity and log-period linear prediction.  The period order itself (sort,
// distinct periods, gaps, prediction ratios) is a plan of T entries computed
// on the host; the device does the B x K x T cell work, one thread per
// (model, period) trace with its K cells.  Every cell is written by its own
// trace's thread only: a distinct period's thread also marks the duplicate
// mismatches that its duplicates see, so no atomics are needed.  All arithmetic
// is rounded operation by operation (no contraction), as in the reference's
// numpy, so the flags are bit-identical.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "modisp_b200.h"

namespace md200 {

// ModeReliabilityFlag bits (python/modisp/reliability.py:12-24)
constexpr uint32_t RF_UNASSESSED = 1, RF_NUMERICAL_FAILURE = 2, RF_ROOT_COUNT_CHANGE = 4, RF_CLOSE_ROOT = 8,
                   RF_RANK_AMBIGUOUS = 16, RF_STEP_JUMP = 32, RF_PREDICTION_MISMATCH = 64,
                   RF_DUPLICATE_MISMATCH = 128, RF_NONFINITE = 256, RF_PERIOD_GAP = 512,
                   RF_SEARCH_UNCERTAIN = 1024;
// trace-flag bits read as failures / as uncertain searches (reliability.py:94-96)
constexpr uint32_t RF_FAILURE_TRACE_BITS = 1u | 4u | 8u | 32u | 64u | 128u | 512u | 1024u;
constexpr uint32_t RF_UNCERTAIN_TRACE_BITS = 2048u | 4096u;

struct ReliabilityArgs {
  const double *v;          // [B][K][T]
  const uint32_t *tflags;   // [B][T] or null (all zero)
  const int64_t *counts;    // [B][T] or null (finite roots per trace)
  const md200_period_plan *plan;  // [T]
  const int32_t *order;     // [T] stable sorted period order
  int B, K, T;
  double close_rtol, max_step, pred_rtol;
  uint16_t *flags;          // [B][K][T]
  uint8_t *assessed;        // [B][K][T]
};

__device__ __forceinline__ bool dup_mismatch(double a, double b) {
  const bool fa = isfinite(a), fb = isfinite(b);
  if (fa != fb) return true;
  return fa && fabs(__dsub_rn(a, b)) > __dmul_rn(1e-10, fmax(a, b));
}

// roots counted for trace (b, t): the caller's counts, else the finite cells
__device__ __forceinline__ int64_t trace_count(const ReliabilityArgs &r, int b, const double *vb, int t) {
  if (r.counts) return r.counts[static_cast<size_t>(b) * r.T + t];
  int64_t n = 0;
  for (int k = 0; k < r.K; ++k) n += isfinite(vb[static_cast<size_t>(k) * r.T + t]);
  return n;
}

__global__ void mode_reliability(ReliabilityArgs r) {
  const size_t gid = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (gid >= static_cast<size_t>(r.B) * r.T) return;
  const int b = static_cast<int>(gid / r.T), t = static_cast<int>(gid - static_cast<size_t>(b) * r.T);
  const int K = r.K, T = r.T;
  const double *vb = r.v + static_cast<size_t>(b) * K * T;
  uint16_t *fb = r.flags + static_cast<size_t>(b) * K * T;
  uint8_t *ab = r.assessed + static_cast<size_t>(b) * K * T;
  const md200_period_plan pl = r.plan[t];
  const uint32_t tf = r.tflags ? r.tflags[static_cast<size_t>(b) * T + t] : 0u;
  const int64_t cnt = trace_count(r, b, vb, t);
  const bool fail = (tf & RF_FAILURE_TRACE_BITS) != 0 || cnt < 0;
  const bool first = (pl.kind & MD200_PLAN_FIRST) != 0, dup = (pl.kind & MD200_PLAN_DUPLICATE) != 0;
  const int prev = pl.prev;
  bool fail_prev = false, changed = false;
  if (!first) {
    const uint32_t tfp = r.tflags ? r.tflags[static_cast<size_t>(b) * T + prev] : 0u;
    const int64_t cntp = trace_count(r, b, vb, prev);
    fail_prev = (tfp & RF_FAILURE_TRACE_BITS) != 0 || cntp < 0;
    changed = cntp != cnt;
    for (int k = 0; k < K && !changed; ++k)
      changed = isfinite(vb[static_cast<size_t>(k) * T + prev]) != isfinite(vb[static_cast<size_t>(k) * T + t]);
  }
  const bool predict = (pl.kind & MD200_PLAN_PREDICT) != 0;
  for (int k = 0; k < K; ++k) {
    const size_t c = static_cast<size_t>(k) * T + t;
    const double x = vb[c];
    const bool fx = isfinite(x);
    uint32_t f = 0;
    if (!fx) f |= RF_NONFINITE;
    if (fail) f |= RF_NUMERICAL_FAILURE;
    if (tf & RF_UNCERTAIN_TRACE_BITS) f |= RF_SEARCH_UNCERTAIN;
    // adjacent ranks (reliability.py:98-105)
    if (k + 1 < K) {
      const double y = vb[c + T], gap = __dsub_rn(y, x);
      if (isfinite(gap)) {
        if (gap <= __dmul_rn(r.close_rtol, y)) f |= RF_CLOSE_ROOT;
        if (gap <= 0.) f |= RF_RANK_AMBIGUOUS;
      }
    }
    if (k > 0) {
      const double w = vb[c - T], gap = __dsub_rn(x, w);
      if (isfinite(gap)) {
        if (gap <= __dmul_rn(r.close_rtol, x)) f |= RF_CLOSE_ROOT;
        if (gap <= 0.) f |= RF_RANK_AMBIGUOUS;
      }
    }
    bool assessed = false;
    if (first) {
      f |= RF_UNASSESSED;
    } else {
      const double a = vb[static_cast<size_t>(k) * T + prev];
      const bool both = isfinite(a) && fx;
      if (changed) f |= RF_ROOT_COUNT_CHANGE;
      if (dup) {
        if (dup_mismatch(a, x)) f |= RF_DUPLICATE_MISMATCH;
        assessed = both && !fail && !fail_prev;
      } else {
        if (pl.kind & MD200_PLAN_GAP) f |= RF_PERIOD_GAP;
        else assessed = both && !fail && !fail_prev;
        if (both && __ddiv_rn(fabs(__dsub_rn(x, a)), fmax(a, x)) > r.max_step) f |= RF_STEP_JUMP;
        if (predict && both) {
          const double o = vb[static_cast<size_t>(k) * T + pl.older];
          if (isfinite(o)) {
            const double predicted = __dadd_rn(a, __dmul_rn(__dsub_rn(a, o), pl.ratio));
            if (fabs(__dsub_rn(x, predicted)) > __dmul_rn(r.pred_rtol, x)) f |= RF_PREDICTION_MISMATCH;
          }
        }
      }
    }
    // this distinct period against each of its duplicates (the reference marks
    // both cells of a mismatching pair)
    if (!dup)
      for (int q = pl.dup_begin; q < pl.dup_end; ++q)
        if (dup_mismatch(x, vb[static_cast<size_t>(k) * T + r.order[q]])) f |= RF_DUPLICATE_MISMATCH;
    fb[c] = static_cast<uint16_t>(f);
    ab[c] = assessed;
  }
  // nearest-rank agreement between the finite roots at prev and at t: a root
  // whose nearest predecessor is another rank, or whose nearest predecessor's
  // nearest successor is another root, is ambiguous (reliability.py:129-135;
  // first minimum on ties, as numpy's argmin)
  if (first || dup) return;
  for (int j = 0; j < K; ++j) {
    const double bj = vb[static_cast<size_t>(j) * T + t];
    if (!isfinite(bj)) continue;
    int ibest = -1;
    double cbest = 0.;
    for (int i = 0; i < K; ++i) {
      const double ai = vb[static_cast<size_t>(i) * T + prev];
      if (!isfinite(ai)) continue;
      const double cost = fabs(__dsub_rn(ai, bj));
      if (ibest < 0 || cost < cbest) { ibest = i; cbest = cost; }
    }
    if (ibest < 0) return;  // no finite root at prev: nothing to compare for any j
    const double ai = vb[static_cast<size_t>(ibest) * T + prev];
    int jbest = -1;
    double dbest = 0.;
    for (int q = 0; q < K; ++q) {
      const double bq = vb[static_cast<size_t>(q) * T + t];
      if (!isfinite(bq)) continue;
      const double cost = fabs(__dsub_rn(ai, bq));
      if (jbest < 0 || cost < dbest) { jbest = q; dbest = cost; }
    }
    if (ibest != j || jbest != j) fb[static_cast<size_t>(j) * T + t] |= RF_RANK_AMBIGUOUS;
  }
}

// The same checks with a trace's roots at t, prev and older held in registers,
// for a mode count fixed at compile time (KM = K; loops unrolled exactly): the
// kernel above reloads them from L1 in every rank comparison and is
// issue-bound.  Same arithmetic, same flags.
template <int KM>
__global__ void __launch_bounds__(256) mode_reliability_small(ReliabilityArgs r) {
  const size_t gid = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (gid >= static_cast<size_t>(r.B) * r.T) return;
  const int b = static_cast<int>(gid / r.T), t = static_cast<int>(gid - static_cast<size_t>(b) * r.T);
  const int K = r.K, T = r.T;
  const double *vb = r.v + static_cast<size_t>(b) * K * T;
  const md200_period_plan pl = r.plan[t];
  const bool first = (pl.kind & MD200_PLAN_FIRST) != 0, dup = (pl.kind & MD200_PLAN_DUPLICATE) != 0;
  const bool predict = (pl.kind & MD200_PLAN_PREDICT) != 0;
  const int prev = first ? t : pl.prev, older = predict ? pl.older : t;
  double x[KM], a[KM], o[KM];
  int nx = 0, na = 0;
#pragma unroll
  for (int k = 0; k < KM; ++k) {
    x[k] = a[k] = o[k] = NAN;
    if (k < K) {
      x[k] = vb[static_cast<size_t>(k) * T + t];
      a[k] = vb[static_cast<size_t>(k) * T + prev];
      if (predict) o[k] = vb[static_cast<size_t>(k) * T + older];
      nx += isfinite(x[k]);
      na += isfinite(a[k]);
    }
  }
  const uint32_t tf = r.tflags ? r.tflags[static_cast<size_t>(b) * T + t] : 0u;
  const int64_t cnt = r.counts ? r.counts[static_cast<size_t>(b) * T + t] : nx;
  const bool fail = (tf & RF_FAILURE_TRACE_BITS) != 0 || cnt < 0;
  bool fail_prev = false, changed = false;
  if (!first) {
    const uint32_t tfp = r.tflags ? r.tflags[static_cast<size_t>(b) * T + prev] : 0u;
    const int64_t cntp = r.counts ? r.counts[static_cast<size_t>(b) * T + prev] : na;
    fail_prev = (tfp & RF_FAILURE_TRACE_BITS) != 0 || cntp < 0;
    changed = cntp != cnt;
#pragma unroll
    for (int k = 0; k < KM; ++k)
      if (k < K && isfinite(a[k]) != isfinite(x[k])) changed = true;
  }
  uint32_t f[KM];
  bool as[KM];
#pragma unroll
  for (int k = 0; k < KM; ++k) {
    f[k] = 0;
    as[k] = false;
    if (k >= K) continue;
    const bool fx = isfinite(x[k]);
    if (!fx) f[k] |= RF_NONFINITE;
    if (fail) f[k] |= RF_NUMERICAL_FAILURE;
    if (tf & RF_UNCERTAIN_TRACE_BITS) f[k] |= RF_SEARCH_UNCERTAIN;
    if (k + 1 < K) {
      const double gap = __dsub_rn(x[k + 1], x[k]);
      if (isfinite(gap)) {
        if (gap <= __dmul_rn(r.close_rtol, x[k + 1])) f[k] |= RF_CLOSE_ROOT;
        if (gap <= 0.) f[k] |= RF_RANK_AMBIGUOUS;
      }
    }
    if (k > 0) {
      const double gap = __dsub_rn(x[k], x[k - 1]);
      if (isfinite(gap)) {
        if (gap <= __dmul_rn(r.close_rtol, x[k])) f[k] |= RF_CLOSE_ROOT;
        if (gap <= 0.) f[k] |= RF_RANK_AMBIGUOUS;
      }
    }
    if (first) {
      f[k] |= RF_UNASSESSED;
    } else {
      const bool both = isfinite(a[k]) && fx;
      if (changed) f[k] |= RF_ROOT_COUNT_CHANGE;
      if (dup) {
        if (dup_mismatch(a[k], x[k])) f[k] |= RF_DUPLICATE_MISMATCH;
        as[k] = both && !fail && !fail_prev;
      } else {
        if (pl.kind & MD200_PLAN_GAP) f[k] |= RF_PERIOD_GAP;
        else as[k] = both && !fail && !fail_prev;
        if (both && __ddiv_rn(fabs(__dsub_rn(x[k], a[k])), fmax(a[k], x[k])) > r.max_step) f[k] |= RF_STEP_JUMP;
        if (predict && both && isfinite(o[k])) {
          const double predicted = __dadd_rn(a[k], __dmul_rn(__dsub_rn(a[k], o[k]), pl.ratio));
          if (fabs(__dsub_rn(x[k], predicted)) > __dmul_rn(r.pred_rtol, x[k])) f[k] |= RF_PREDICTION_MISMATCH;
        }
      }
    }
  }
  if (!dup)
    for (int q = pl.dup_begin; q < pl.dup_end; ++q) {
      const int td = r.order[q];
#pragma unroll
      for (int k = 0; k < KM; ++k)
        if (k < K && dup_mismatch(x[k], vb[static_cast<size_t>(k) * T + td])) f[k] |= RF_DUPLICATE_MISMATCH;
    }
  if (!first && !dup && na > 0) {
    // nearest-rank agreement (first minimum on ties, as numpy's argmin)
#pragma unroll
    for (int j = 0; j < KM; ++j) {
      if (j >= K || !isfinite(x[j])) continue;
      int ibest = -1;
      double cbest = 0., abest = 0.;
#pragma unroll
      for (int i = 0; i < KM; ++i) {
        if (i >= K || !isfinite(a[i])) continue;
        const double cost = fabs(__dsub_rn(a[i], x[j]));
        if (ibest < 0 || cost < cbest) { ibest = i; cbest = cost; abest = a[i]; }
      }
      int jbest = -1;
      double dbest = 0.;
#pragma unroll
      for (int q = 0; q < KM; ++q) {
        if (q >= K || !isfinite(x[q])) continue;
        const double cost = fabs(__dsub_rn(abest, x[q]));
        if (jbest < 0 || cost < dbest) { jbest = q; dbest = cost; }
      }
      if (ibest != j || jbest != j) f[j] |= RF_RANK_AMBIGUOUS;
    }
  }
  uint16_t *fb = r.flags + static_cast<size_t>(b) * K * T;
  uint8_t *ab = r.assessed + static_cast<size_t>(b) * K * T;
#pragma unroll
  for (int k = 0; k < KM; ++k)
    if (k < K) {
      fb[static_cast<size_t>(k) * T + t] = static_cast<uint16_t>(f[k]);
      ab[static_cast<size_t>(k) * T + t] = as[k];
    }
}

}  // namespace md200
