// split_scan.cuh -- the single-precision scan as rounds of separate kernels.
//
// The fused scan (scan<float, WAVE>) runs one trace per warp from start to end:
// each 32-sample step computes positions, evaluates them, re-evaluates the
// sign-uncertain ones in FP64 and does the bookkeeping, all latency-bound
// work of one warp.  Here the same steps run as rounds over an active set of
// traces, each stage with the parallel shape that suits it:
//   split_feed_count/fill  the active set refilled from the trace list (new
//                          traces start from scan_start)
//   split_positions        one warp per trace: the next SPLIT_STEPS steps'
//                          positions, merged exactly as the fused scan merges
//                          them (scan_positions, scan_position32)
//   split_eval32           one thread per sample: the FP32 secular value; the
//                          near-cutoff band takes the trace's FP64 tail values;
//                          sign-uncertain samples are listed for FP64
//   split_eval32_pair      Rayleigh: the same with one thread per two samples of
//                          a trace, evaluated together in paired FP32
//                          instructions (sm_100 .f32x2)
//   split_redo             one thread per listed sample: its FP64 value
//   split_book             one thread per trace: the samples in order through
//                          the fused scan's bookkeeping (sign changes, regular
//                          samples, trough tests), brackets appended; a trough
//                          that needs a window pauses the trace at that sample,
//                          the last cell of a finished trace is requested too
//   split_zoom             one warp per request: the FP32 screen and the FP64
//                          zoom of a trough window (screen_trough32,
//                          zoom_trough), or the last cell (last_cell)
// Every sample goes through the same arithmetic and every decision through the
// same rule as in the fused scan, in the same order, so the brackets -- and the
// roots -- are the fused scan's bit for bit.  The state between rounds is the
// fused scan's ScanState; a paused trace resumes from its cursors (the samples
// after the pause are positioned and evaluated again).  Traces still unfinished
// after the last round, and any the rounds never reached, are finished by the
// fused kernel (resume mode).
#pragma once
#include "kernels.cuh"

namespace md200 {

// Compile-time tuning: 32-sample steps per trace per round (two measured best:
// fewer samples evaluated past a trace's last bracket than four, half the
// rounds of one); the evaluation kernel's minimum resident CTAs per SM (1: no
// register cap; capping it measured no faster); Rayleigh values two samples
// per thread in paired FP32 instructions (split_eval32_pair, on with two steps
// per round), that kernel's minimum resident CTAs per SM (4: 122 registers,
// no spills; uncapped, 138 registers and 3 CTAs ran 13 % slower, 5 CTAs spill)
// and its grid in CTAs per SM (64: 2.4 % faster than 16, 128 no faster; the
// grid-stride loop then takes a few pairs per thread).
#ifndef MD200_SPLIT_STEPS
#define MD200_SPLIT_STEPS 2
#endif
#ifndef MD200_SPLIT_EVAL_BLOCKS
#define MD200_SPLIT_EVAL_BLOCKS 1
#endif
#ifndef MD200_SPLIT_PAIR
#define MD200_SPLIT_PAIR (MD200_SPLIT_STEPS == 2)
#endif
#ifndef MD200_SPLIT_PAIR_BLOCKS
#define MD200_SPLIT_PAIR_BLOCKS 4
#endif
#ifndef MD200_SPLIT_PAIR_GRID
#define MD200_SPLIT_PAIR_GRID 64
#endif
constexpr int SPLIT_STEPS = MD200_SPLIT_STEPS;    // 32-sample steps per trace per round
constexpr int SPLIT_SAMPLES = 32 * SPLIT_STEPS;  // sample slots per active trace
constexpr int SPLIT_ACTIVE_MAX = 1 << 20;         // active-set capacity (traces)
constexpr int SPLIT_MIN_TRACES = 4096;            // runs with fewer traces use the fused kernel
constexpr unsigned SK_SEED = 1, SK_NEAR = 2, SK_EXACT = 4, SK_REDO = 8;
constexpr int ZOOM_TROUGH = 0, ZOOM_LAST = 1;

}  // namespace md200

// One sample of a round: position, secular value, shape feature and
// log-magnitude, bits (seed, near cutoff, FP64 value).  32 bytes, one memory
// sector: the bookkeeping thread of a trace reads its samples one sector each.
// The trough tests and windows take the shape feature and log-magnitude in
// single precision only, so float keeps every decision of the fused scan.
struct md200::SplitSample {
  double c, F;
  float g, M;
  unsigned k, pad;
};

// An active trace's constants for the evaluation threads, written by its
// positions warp: one load instead of the chain trace -> model -> table.
struct md200::SplitTrace {
  double w;
  int t, b, L, water, pad0, pad1;
};

namespace md200 {
static_assert(sizeof(SplitSample) == 32, "one sector per sample");

// Warp-aggregated append: every lane of the warp calls it (n = 0 where there is
// nothing to add); returns this lane's base index in the list behind `counter`.
__device__ __forceinline__ int warp_append(int *counter, int n, int lane) {
  int incl = n;
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(FULL, incl, o);
    if (lane >= o) incl += v;
  }
  const int total = __shfl_sync(FULL, incl, 31);
  int base = 0;
  if (lane == 31 && total) base = atomicAdd(counter, total);
  base = __shfl_sync(FULL, base, 31);
  return base + incl - n;
}

__device__ __forceinline__ void split_count(const Dev &d, unsigned long long evals, unsigned long long evals32,
                                            unsigned long long steps, unsigned long long steps32, int lane) {
  if (!d.stats) return;
  for (int o = 16; o; o >>= 1) {
    evals += __shfl_xor_sync(FULL, evals, o);
    evals32 += __shfl_xor_sync(FULL, evals32, o);
    steps += __shfl_xor_sync(FULL, steps, o);
    steps32 += __shfl_xor_sync(FULL, steps32, o);
  }
  if (lane == 0) {
    if (evals) atomicAdd(&d.stats[0], evals);
    if (evals32) atomicAdd(&d.stats[1], evals32);
    if (steps) atomicAdd(&d.stats[2], steps);
    if (steps32) atomicAdd(&d.stats[3], steps32);
  }
}

// ---------------------------------------------------------------------------
// The active set of round r lives in sp_act[p], p = r & 1; traces that go on to
// the next round are appended to sp_act[1 - p].
// ---------------------------------------------------------------------------
__global__ void split_feed_count(Dev d, int p) {
  int *c = d.ctr;
  const int n_act = c[C_SP_ACT0 + p], n_list = c[C_NTRACE], feed = c[C_SP_FEED];
  const int room = d.sp_cap - n_act, left = n_list - feed;
  const int take = room < left ? room : left;
  c[C_SP_BASE] = n_act;
  c[C_SP_TAKE] = take;
  c[C_SP_ACT0 + p] = n_act + take;
  c[C_SP_FEED] = feed + take;
  c[C_SP_ACT0 + 1 - p] = 0;
  c[C_SP_REDO] = 0;
  c[C_SP_ZOOM] = 0;
}

__global__ void split_feed_fill(Dev d, int p) {
  const int base = d.ctr[C_SP_BASE], take = d.ctr[C_SP_TAKE];
  const int first = d.ctr[C_SP_FEED] - take;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < take; i += gridDim.x * blockDim.x) {
    const int t = d.trace_list[first + i];
    d.sp_act[p][base + i] = t;
    d.sp_state[t] = scan_start(d, trace_ctx(d, t));
    d.sp_kf[t] = 0;
  }
}

// One warp per active trace: positions of its next SPLIT_STEPS steps from the
// state's cursors.  Slots past the window hold INFINITY.
__global__ void __launch_bounds__(128) split_positions(Dev d, int p) {
  __shared__ double mbuf_all[4][32];
  __shared__ unsigned char kbuf_all[4][32];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  double *mbuf = mbuf_all[wib];
  unsigned char *kbuf = kbuf_all[wib];
  const int n = d.ctr[C_SP_ACT0 + p];
  const double step = 1. / d.density;
  for (int i = blockIdx.x * 4 + wib; i < n; i += gridDim.x * 4) {
    const int t = d.sp_act[p][i];
    const TraceCtx x = trace_ctx(d, t);
    ScanState st = d.sp_state[t];
    // the knot interval of the round's first grid point: no later target of this
    // trace lies below it (consumed samples only move the cursors up)
    int kfrom = d.sp_kf[t];
    if (lane == 0) {
      SplitTrace tr;
      tr.w = x.w;
      tr.t = t;
      tr.b = x.b;
      tr.L = d.mL[x.b];
      tr.water = d.mwater[x.b];
      tr.pad0 = tr.pad1 = 0;
      d.sp_tr[i] = tr;
    }
    SplitSample *ss = d.sp_s + static_cast<size_t>(i) * SPLIT_SAMPLES;
    bool done = false;
    for (int s = 0; s < SPLIT_STEPS; ++s) {
      double c = INFINITY;
      unsigned seeds = 0;
      if (!done) {
        const unsigned vm = scan_positions<true>(x, st, step, lane, mbuf, kfrom, c, kbuf, &seeds);
        done = vm == 0;
        if (s == 0 && lane == 0) d.sp_kf[t] = kfrom;
      }
      unsigned k = 0;
      if (c < INFINITY) {
        bool near_cut;
        scan_position32(c, x.hi, near_cut);
        k = ((seeds >> lane) & 1u ? SK_SEED : 0u) | (near_cut ? SK_NEAR : 0u);
      }
      ss[s * 32 + lane].c = c;
      ss[s * 32 + lane].k = k;
    }
  }
}

// A near-cutoff sample: the trace's FP64 tail value when it is at this position
// (returns false), else true (the sample goes to the FP64 list).
__device__ __forceinline__ bool split_near(const Dev &d, int t, SplitSample &smp, double c, unsigned &k) {
  const double4 *tail = d.tail + 2 * static_cast<size_t>(t);
  const double4 t0 = tail[0], t1 = tail[1];
  const double4 tv = c == t0.x ? t0 : t1;
  if (c == tv.x && isfinite(tv.y)) {
    smp.F = tv.y;
    smp.g = static_cast<float>(tv.z);
    smp.M = static_cast<float>(tv.w);
    k |= SK_EXACT;
    return false;
  }
  return true;
}

// One thread per sample slot: the FP32 value (the fused scan's scan_eval call on
// the same single-precision position), or the trace's FP64 tail value in the
// near-cutoff band; samples the FP32 value leaves sign-uncertain, and near-cutoff
// samples without a tail value, are listed for FP64 (scan_complete32's rule).
template <int WAVE>
__global__ void __launch_bounds__(128, MD200_SPLIT_EVAL_BLOCKS) split_eval32(Dev d, int p) {
  const int lane = threadIdx.x & 31;
  const long long n = static_cast<long long>(d.ctr[C_SP_ACT0 + p]) * SPLIT_SAMPLES;
  const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
  unsigned long long steps = 0;  // FP32 layer steps evaluated here (MD200_STAT_SPLIT_EVAL_STEPS)
  // the loop runs whole warps (n is a multiple of 32), so appends are warp-wide
  for (long long q = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; q < n; q += stride) {
    const int i = static_cast<int>(q / SPLIT_SAMPLES);
    SplitSample &smp = d.sp_s[q];
    const double c = smp.c;
    unsigned k = smp.k;
    bool redo = false;
    if (c < INFINITY) {
      const SplitTrace tr = d.sp_tr[i];
      if (k & SK_NEAR) {
        redo = split_near(d, tr.t, smp, c, k);
      } else {
        const LayerView<float> view = make_view<float>(layer_table<float>(d, tr.b), d.Ls, tr.L, tr.water);
        const float c32 = static_cast<float>(c);
        float F32, g32, M32;
        scan_eval<float, WAVE, 1>(view, static_cast<float>(tr.w), &c32, &F32, &g32, &M32);
        steps += layer_steps(tr.L, tr.water);
        const double g = g32;
        smp.F = F32;
        smp.g = g32;
        smp.M = M32;
        redo = !(fabs(g) > MD200_REDO_G);
      }
      if (!redo) smp.k = k;
    }
    const int at = warp_append(&d.ctr[C_SP_REDO], redo ? 1 : 0, lane);
    if (redo) d.sp_redo[at] = static_cast<int>(q);
  }
  if (d.stats) {
    for (int o = 16; o; o >>= 1) steps += __shfl_xor_sync(FULL, steps, o);
    if (lane == 0 && steps) atomicAdd(&d.stats[19], steps);
  }
}

#if MD200_SPLIT_PAIR
// Rayleigh: one thread per pair of sample slots of an active trace -- slot j of
// its first 32-sample step and slot j of its second -- whose FP32 values come
// from one paired evaluation (rayleigh_eval32<R2>: each half bit for bit the
// single evaluation split_eval32 and the fused scan make).  A slot past the
// window or in the near-cutoff band leaves its half to a copy of the other
// sample, whose result is not stored.
static_assert(SPLIT_SAMPLES == 64, "the paired evaluation takes the two 32-sample steps of a round");
__global__ void __launch_bounds__(128, MD200_SPLIT_PAIR_BLOCKS) split_eval32_pair(Dev d, int p) {
  const int lane = threadIdx.x & 31;
  const long long n = static_cast<long long>(d.ctr[C_SP_ACT0 + p]) * 32;
  const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
  unsigned long long steps = 0;
  // whole warps run the loop (n and stride are multiples of 32): appends are warp-wide
  for (long long q = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; q < n; q += stride) {
    const int i = static_cast<int>(q >> 5);
    const long long q0 = static_cast<long long>(i) * SPLIT_SAMPLES + (q & 31), q1 = q0 + 32;
    SplitSample &s0 = d.sp_s[q0], &s1 = d.sp_s[q1];
    const double c0 = s0.c, c1 = s1.c;
    unsigned k0 = s0.k, k1 = s1.k;
    bool redo0 = false, redo1 = false;
    if (c0 < INFINITY || c1 < INFINITY) {
      const SplitTrace tr = d.sp_tr[i];
      const bool e0 = c0 < INFINITY && !(k0 & SK_NEAR), e1 = c1 < INFINITY && !(k1 & SK_NEAR);
      if (c0 < INFINITY && !e0) redo0 = split_near(d, tr.t, s0, c0, k0);
      if (c1 < INFINITY && !e1) redo1 = split_near(d, tr.t, s1, c1, k1);
      if (e0 || e1) {
        const LayerView<float> view = make_view<float>(layer_table<float>(d, tr.b), d.Ls, tr.L, tr.water);
        const float w = static_cast<float>(tr.w);
        const float x0 = static_cast<float>(e0 ? c0 : c1), x1 = static_cast<float>(e1 ? c1 : c0);
        const float2 kk = make_float2(w / x0, w / x1);
        float2 F, g, M;
        rayleigh_eval32<R2>(view, kk, make_float2(w / kk.x, w / kk.y), w, &F, &g, &M);
        const unsigned long long ls = layer_steps(tr.L, tr.water);
        if (e0) {
          s0.F = F.x;
          s0.g = g.x;
          s0.M = M.x;
          redo0 = !(fabs(static_cast<double>(g.x)) > MD200_REDO_G);
          steps += ls;
        }
        if (e1) {
          s1.F = F.y;
          s1.g = g.y;
          s1.M = M.y;
          redo1 = !(fabs(static_cast<double>(g.y)) > MD200_REDO_G);
          steps += ls;
        }
      }
      if (c0 < INFINITY && !redo0) s0.k = k0;
      if (c1 < INFINITY && !redo1) s1.k = k1;
    }
    int at = warp_append(&d.ctr[C_SP_REDO], (redo0 ? 1 : 0) + (redo1 ? 1 : 0), lane);
    if (redo0) d.sp_redo[at++] = static_cast<int>(q0);
    if (redo1) d.sp_redo[at] = static_cast<int>(q1);
  }
  if (d.stats) {
    for (int o = 16; o; o >>= 1) steps += __shfl_xor_sync(FULL, steps, o);
    if (lane == 0 && steps) atomicAdd(&d.stats[19], steps);
  }
}
#endif  // MD200_SPLIT_PAIR

// One thread per listed sample: its FP64 value (eval64_outline, as in the fused
// scan).
template <int WAVE>
__global__ void __launch_bounds__(128) split_redo(Dev d, int p) {
  const int n = d.ctr[C_SP_REDO];
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const int q = d.sp_redo[r];
    const SplitTrace tr = d.sp_tr[q / SPLIT_SAMPLES];
    SplitSample &smp = d.sp_s[q];
    double g, M;
    const double F = eval64_outline(make_view<double>(layer_table<double>(d, tr.b), d.Ls, tr.L, tr.water), WAVE,
                                    tr.w, smp.c, &g, &M);
    smp.F = F;
    smp.g = static_cast<float>(g);
    smp.M = static_cast<float>(M);
    smp.k |= SK_EXACT | SK_REDO;
  }
}

// A finished trace's brackets published for refinement (scan_finish without
// the last cell), one thread per trace; every lane of the warp calls it.
__device__ __forceinline__ void split_publish(const Dev &d, int t, const ScanState &st, bool publish, int lane) {
  int n = 0;
  if (publish) {
    d.nbr[t] = st.nbr;
    if (st.tfl) atomicOr(&d.tflags[t], st.tfl);
    if (!(st.tfl & TRACE_SEARCH_UNCONVERGED)) n = st.nbr;
  }
  const int base = warp_append(&d.ctr[C_NREFINE], n, lane);
  for (int k = 0; k < n; ++k) d.refine_list[base + k] = t * d.KB + k;
}

// Does a finished trace need its last cell examined (scan_finish's condition)?
// -- and does the shape feature fall into the window end steeply enough that
// last_cell would screen the cell (its first test, evaluated here so that only
// those traces take a warp)?
__device__ __forceinline__ bool needs_last_cell(const ScanState &st, int K) {
  if (!((st.bits & SS_FINISHED) && st.nbr < K && !(st.tfl & TRACE_SEARCH_UNCONVERGED) && (st.bits & SS_HR1) &&
        (st.bits & SS_HR2) && st.R2.c < st.R1.c && st.zoom_right <= st.R2.c &&
        sample_segment(st.R1) == sample_segment(st.R2)))
    return false;
  const double sgn = sample_sign(st.R1);
  const float u = static_cast<float>(sgn) * st.R2.g, v = static_cast<float>(sgn) * st.R1.g;
  const float h0 = static_cast<float>(st.R1.c - st.R2.c);
  const float noise = pair_noise(true, st.R2, st.R1);
  return u > v + noise && v / ((u - v) / h0) < 1.25f * h0;
}

// One thread per active trace: its samples of this round in order, through the
// bookkeeping of scan_bookkeep (one lane's share of it, carried sample by
// sample).  Ends at the trace's K-th bracket, at the end of its window, at a
// non-finite value, at a trough that needs a window (paused there), or at the
// end of the round's samples (continued next round).
template <int WAVE>
__global__ void __launch_bounds__(128) split_book(Dev d, int p) {
  constexpr bool single = true;
  const int lane = threadIdx.x & 31;
  const int n = d.ctr[C_SP_ACT0 + p];
  const int stride = gridDim.x * blockDim.x;
  const int n_pad = (n + 31) & ~31;
  // counters of the samples the bookkeeping consumes, as the fused scan counts
  // its steps' samples: each an FP32 evaluation, the re-evaluated ones also FP64
  unsigned long long ev = 0, ev32 = 0, sts = 0, sts32 = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_pad; i += stride) {
    const bool active = i < n;
    int t = 0;
    ScanState st;
    int K = 0;
    bool go_on = false, publish = false, zoom = false;
    int ztype = ZOOM_TROUGH;
    if (active) {
      t = d.sp_act[p][i];
      st = d.sp_state[t];
      K = d.tr_modes[t] + 2;
      double *slot = d.slot + static_cast<size_t>(t) * d.KB * SLOT;
      const size_t base = static_cast<size_t>(i) * SPLIT_SAMPLES;
      const SplitTrace tr = d.sp_tr[i];
      const unsigned long long nsteps = layer_steps(tr.L, tr.water);
      bool stop = false;  // the K-th bracket, the window end or a non-finite value
      // the next record is loaded while this one is worked on (the loop is a
      // chain of dependent decisions; its loads need not be)
      SplitSample ahead = d.sp_s[base];
      for (int j = 0; j < SPLIT_SAMPLES; ++j) {
        const SplitSample smp = ahead;
        if (j + 1 < SPLIT_SAMPLES) ahead = d.sp_s[base + j + 1];
        const double c = smp.c;
        if (!(c < INFINITY)) {  // the window is exhausted
          st.bits |= SS_FINISHED;
          stop = true;
          break;
        }
        const double F = smp.F;
        const float gf = smp.g, Mf = smp.M;
        const double g = gf;
        const unsigned k = smp.k;
        const bool exact = (k & SK_EXACT) != 0;
        ++ev32;
        sts32 += nsteps;
        ev += (k & SK_REDO) ? 2 : 1;
        sts += (k & SK_REDO) ? 2 * nsteps : nsteps;
        if (!(isfinite(F) && isfinite(g))) {
          st.tfl |= TRACE_NONFINITE | TRACE_SEARCH_UNCONVERGED;
          st.bits |= SS_FINISHED;
          stop = true;
          break;
        }
        // sign change against the previous sample
        const bool vl = (st.bits & SS_HAVE1) != 0;
        const double cl = st.c1, Fl = st.F1;
        const bool exl = (st.bits & SS_EX1) != 0;
        const bool sc = vl && (signbit(Fl) != signbit(F));
        const int myseg = st.nseg + (sc ? 1 : 0);
        const Sample me{c, gf, Mf, myseg | (exact ? (1 << 29) : 0) | (signbit(F) ? (1 << 30) : 0)};
        const bool reg = !(vl && c - cl < 1e-6 * c);
        const Sample P1 = st.R1, P2 = st.R2;
        const bool hp1 = (st.bits & SS_HR1) != 0, hp2 = (st.bits & SS_HR2) != 0;
        bool tr = false, trm = false;
        if (reg && hp1 && hp2 && sample_segment(P2) == myseg && sample_segment(P1) == myseg) {
          const double sgn = sample_sign(P1);
          tr = trough_may_hide_roots(P2.c, P1.c, c, sgn * P2.g, sgn * P1.g, sgn * gf, pair_noise(single, P2, P1),
                                     pair_noise(single, P1, me));
          if (!tr) trm = magnitude_dip(P2.c, P1.c, c, P2.M, P1.M, Mf) > MDIP;
          tr = tr || trm;
        }
        bool pause = false;
        if (sc) {
          if (st.nbr < K) {
            put_bracket(slot, st.nbr, cl, c, exl ? Fl : NAN, exact ? F : NAN);
            ++st.nbr;
          }
        } else if (tr && st.nbr < K) {
          double x0 = P2.c, sa, ma;
          const double x1 = P1.c, x2 = c;
          const double sgn = sample_sign(P1);
          sa = sgn * P2.g;
          ma = P2.M;
          if (x0 < st.zoom_right) {  // overlaps the previous window: start at its middle sample
            x0 = x1;
            sa = sgn * P1.g;
            ma = P1.M;
          }
          st.zoom_right = x2;
          double *za = d.sp_zarg + static_cast<size_t>(i) * 8;
          za[0] = x0;
          za[1] = x2;
          za[2] = sa;
          za[3] = sgn * g;
          za[4] = ma;
          za[5] = Mf;
          za[6] = sgn;
          za[7] = trm ? 1. : 0.;
          pause = true;
        }
        // carries
        st.nseg = myseg;
        st.c1 = c;
        st.F1 = F;
        st.bits = (st.bits & ~SS_EX1) | SS_HAVE1 | (exact ? SS_EX1 : 0);
        if (reg) {
          st.R2 = st.R1;
          st.bits = (st.bits & ~SS_HR2) | ((st.bits & SS_HR1) ? SS_HR2 : 0);
          st.R1 = me;
          st.bits |= SS_HR1;
        }
        if (k & SK_SEED) ++st.si;
        else ++st.gi;
        if (pause) {
          zoom = true;
          ztype = ZOOM_TROUGH;
          break;
        }
        if (st.nbr >= K) {
          stop = true;
          break;
        }
      }
      if (stop) {
        if (needs_last_cell(st, K)) {
          zoom = true;
          ztype = ZOOM_LAST;
        } else {
          publish = true;
        }
      } else if (!zoom) {
        go_on = true;  // the round's samples are used up: more next round
      }
      d.sp_state[t] = st;
    }
    split_publish(d, t, st, publish, lane);
    const int za = warp_append(&d.ctr[C_SP_ZOOM], zoom ? 1 : 0, lane);
    if (zoom) d.sp_zoom[za] = ztype == ZOOM_LAST ? -(i + 1) : i;
    const int ga = warp_append(&d.ctr[C_SP_ACT0 + 1 - p], go_on ? 1 : 0, lane);
    if (go_on) d.sp_act[1 - p][ga] = t;
  }
  split_count(d, ev, ev32, sts, sts32, lane);
}

// One warp per window request: a trough window (screened in FP32, zoomed in
// FP64 unless dismissed) after which the trace goes on, or the last cell of a
// finished trace, after which it is published.
template <int WAVE>
__global__ void __launch_bounds__(128) split_zoom(Dev d, int p) {
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int n = d.ctr[C_SP_ZOOM];
  for (int r = blockIdx.x * (blockDim.x >> 5) + wib; r < n; r += gridDim.x * (blockDim.x >> 5)) {
    const int code = d.sp_zoom[r];
    const bool last = code < 0;
    const int i = last ? -code - 1 : code;
    const int t = d.sp_act[p][i];
    const TraceCtx x = trace_ctx(d, t);
    ScanState st = d.sp_state[t];
    const LayerView<float> view = make_view<float>(layer_table<float>(d, x.b), d.Ls, d.mL[x.b], d.mwater[x.b]);
    const LayerView<double> view64 = global_view(d, x.b);
    unsigned long long ev = 0, ev32 = 0, s = 0, s32 = 0, zooms = 0;
    if (last) {
      st.nbr = last_cell<float, WAVE>(view, view64, x.w, st.R2, st.R1, d.tol, x.slot, st.nbr, x.K, lane, x.nsteps,
                                      ev, ev32, s, s32, zooms);
    } else {
      const double *za = d.sp_zarg + static_cast<size_t>(i) * 8;
      const double x0 = za[0], x2 = za[1], sa = za[2], sb = za[3], ma = za[4], mb = za[5], sgn = za[6];
      const int mode = za[7] != 0. ? 1 : 0;
      unsigned long long se = 0;
      const bool dismissed = screen_trough32<WAVE>(view, static_cast<float>(x.w), x0, x2, sa, sb, ma, mb, sgn, mode,
                                                   lane, se);
      ev += se;
      ev32 += se;
      s += se * x.nsteps;
      s32 += se * x.nsteps;
      if (!dismissed) {
        unsigned long long ze = 0;
        st.nbr = zoom_trough<WAVE>(view64, x.w, x0, x2, sa, sb, ma, mb, sgn, mode, d.tol, x.slot, st.nbr, x.K, lane,
                                   ze);
        ev += ze;
        s += ze * x.nsteps;
        ++zooms;
      }
    }
    __syncwarp();
    if (lane == 0) {
      if (d.stats) {
        if (ev) atomicAdd(&d.stats[0], ev);
        if (ev32) atomicAdd(&d.stats[1], ev32);
        if (s) atomicAdd(&d.stats[2], s);
        if (s32) atomicAdd(&d.stats[3], s32);
        if (zooms) atomicAdd(&d.stats[5], zooms);
      }
      d.sp_state[t] = st;
      if (last || st.nbr >= x.K) {
        d.nbr[t] = st.nbr;
        if (st.tfl) atomicOr(&d.tflags[t], st.tfl);
      } else {
        d.sp_act[1 - p][atomicAdd(&d.ctr[C_SP_ACT0 + 1 - p], 1)] = t;
      }
    }
    if (last || st.nbr >= x.K) {
      int base = 0;
      if (lane == 0 && !(st.tfl & TRACE_SEARCH_UNCONVERGED)) base = atomicAdd(&d.ctr[C_NREFINE], st.nbr);
      base = __shfl_sync(FULL, base, 0);
      if (!(st.tfl & TRACE_SEARCH_UNCONVERGED))
        for (int k = lane; k < st.nbr; k += 32) d.refine_list[base + k] = t * d.KB + k;
    }
    __syncwarp();
  }
}

}  // namespace md200
