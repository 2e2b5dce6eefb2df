// kernels.cuh -- the engine's CUDA kernels (sm_100a).
//
// Pipeline per run (one stream, no host synchronisation between stages):
//   prep_models   one warp per model: drop zero-thickness padding rows, prepare
//                 reciprocals in FP64 and FP32 tables, search window, the
//                 phase-count knot table that shapes the scan grid, seed points
//   init_traces   trace list (period-major: the costly short periods first)
//   scan<T>       persistent, one warp per trace: 32 grid points per step,
//                 secular value + shape feature in precision T, sign changes
//                 by warp ballot, compaction into bracket slots in velocity
//                 order; a same-sign trough of the shape feature (a possible
//                 hidden close pair) is zoomed into by the whole warp in FP64;
//                 sign-uncertain FP32 samples are re-evaluated in FP64
//   refine        one bracket per lane, lanes refilled from the bracket list:
//                 FP64 endpoint confirmation (FP32 scans) and FP64 Brent
//                 refinement on scale-consistent samples, ending on the secant
//                 point of the converged bracket
//   [FP32 only] collect_repairs + scan<double>/refine on the traces whose
//                 FP32 brackets FP64 did not confirm
//   assemble      one thread per trace: order, cap and write the roots, flags,
//                 counts and group-velocity windows
//   group         one thread per root: FP64 group velocity from forward-mode
//                 derivatives dF/dk and dF/domega of the secular function
//   [FP32 only] continuity_screen + scan<double>/refine/assemble/group on the
//                 traces whose roots break the bilateral envelope of their
//                 neighbouring periods
// Outside the run: root_jacobians (adjoint.cuh) and mode_reliability
// (reliability.cuh) work on a run's results.
#pragma once
#include "engine.cuh"
#include "secular.cuh"

namespace md200 {

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// 16-byte asynchronous global->shared copy (Ampere+ cp.async, bypassing L1).
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::);
}

template <class T>
__device__ __forceinline__ const T *layer_table(const Dev &d, int b);
template <>
__device__ __forceinline__ const double *layer_table<double>(const Dev &d, int b) {
  return d.layer64 + static_cast<size_t>(b) * ROWS * d.Ls;
}
template <>
__device__ __forceinline__ const float *layer_table<float>(const Dev &d, int b) {
  return d.layer32 + static_cast<size_t>(b) * ROWS * d.Ls;
}

template <class T>
__device__ __forceinline__ LayerView<T> make_view(const T *tab, int Ls, int L, int water) {
  LayerView<T> v;
  v.base = tab;
  v.Ls = Ls;
  v.L = L;
  v.water = water;
  return v;
}

// Out-of-line secular evaluation for the scan: the scan's bookkeeping is saved
// once per 32-sample step around the call instead of competing with the layer
// recurrence for registers.
template <class T, int WAVE, int S>
__device__ __noinline__ void scan_eval(const LayerView<T> view, T w, const T *c, T *F, T *g, T *lm) {
  T k[S];
#pragma unroll
  for (int s = 0; s < S; ++s) k[s] = w / c[s];
  secular_multi<T, T, S, WAVE>(view, k, w, F, g, lm);
}

// Layer recurrence steps of one evaluation.
__device__ __forceinline__ int layer_steps(int L, int water) { return L - 1 - water; }

// FP64 secular value (and shape feature) from a global-memory table.
__device__ __forceinline__ double eval64(const LayerView<double> &m, int wave, double w, double c,
                                         double *g) {
  return secular<double, double>(m, wave, w / c, w, g);
}

// Out-of-line FP64 evaluation for the rare FP64 re-evaluations inside the FP32
// scan, so their registers do not weigh on the single-precision loop.
__device__ __noinline__ double eval64_outline(const LayerView<double> &m, int wave, double w, double c,
                                              double *g, double *lm) {
  return secular<double, double>(m, wave, w / c, w, g, lm);
}

// Rayleigh-wave speed of a homogeneous half-space by bisection of the
// Rayleigh cubic (cpp/common/physics.hpp:140-144).  Every operation is rounded
// separately (no FMA contraction), matching the reference's -ffp-contract=off
// build bit for bit: the search window is reported and compared exactly.
__device__ double rayleigh_speed(double vp, double vs) {
  const double q = __ddiv_rn(vs, vp), ratio = __dmul_rn(q, q);
  double l = 0., h = 1.;
  for (int j = 0; j < 56; ++j) {
    const double x = __dmul_rn(__dadd_rn(l, h), .5);
    const double a = __dadd_rn(__dmul_rn(__dadd_rn(x, -8.), x), 24.);
    const double f = __dadd_rn(__dmul_rn(__dadd_rn(a, -__dmul_rn(16., ratio)), x),
                               -__dmul_rn(16., __dadd_rn(1., -ratio)));
    if (f < 0.) l = x; else h = x;
  }
  return __dmul_rn(vs, __dsqrt_rn(__dmul_rn(__dadd_rn(l, h), .5)));
}

// Scholte-wave speed of a fluid over a solid half-space by bisection
// (cpp/common/physics.hpp:146-156), separately rounded like rayleigh_speed.
__device__ double scholte_speed(double vf, double rf, double vp, double vs, double rs) {
  const double q1 = __ddiv_rn(vs, vp), ratio = __dmul_rn(q1, q1);
  const double q2 = __ddiv_rn(vs, vf), qf = __dmul_rn(q2, q2);
  double l = 0., h = fmax(0., __dmul_rn(fmin(1., __ddiv_rn(vf, vs)), __dadd_rn(1., -1e-12)));
  for (int j = 0; j < 64; ++j) {
    const double x = __dmul_rn(__dadd_rn(l, h), .5), x2 = __dmul_rn(x, x);
    const double A = __dsqrt_rn(fmax(0., __dadd_rn(1., -__dmul_rn(ratio, x2))));
    const double B = __dsqrt_rn(fmax(0., __dadd_rn(1., -x2)));
    const double num = __dmul_rn(4., __dadd_rn(__dadd_rn(1., ratio), -__dmul_rn(ratio, x2)));
    const double t1 = __ddiv_rn(num, __dadd_rn(1., __dmul_rn(A, B)));
    const double t2 = __ddiv_rn(__dmul_rn(__dmul_rn(__ddiv_rn(rf, rs), x2), A),
                                __dsqrt_rn(fmax(1e-30, __dadd_rn(1., -__dmul_rn(qf, x2)))));
    const double f = __dadd_rn(__dadd_rn(__dadd_rn(t1, -4.), x2), t2);
    if (f < 0.) l = x; else h = x;
  }
  return __dmul_rn(vs, __dmul_rn(__dadd_rn(l, h), .5));
}

// Warp-cooperative bitonic sort of n2 (a power of two) keys with int payloads.
__device__ void warp_bitonic(double *key, int *val, int n2, int lane) {
  for (int size = 2; size <= n2; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = lane; i < (n2 >> 1); i += 32) {
        const int lo = 2 * i - (i & (stride - 1));
        const int hi = lo + stride;
        const bool up = (lo & size) == 0;
        const double a = key[lo], b = key[hi];
        if ((a > b) == up) {
          key[lo] = b;
          key[hi] = a;
          const int t = val[lo];
          val[lo] = val[hi];
          val[hi] = t;
        }
      }
      __syncwarp();
    }
  }
}

__device__ __forceinline__ int pow2_ceil(int n) {
  int p = 1;
  while (p < n) p <<= 1;
  return p;
}

// Phase-count density N(c) = 2 sum_j h_j sqrt(1/v_j^2 - 1/c^2) over the finite
// layers, S waves (and P waves for Rayleigh) (cpp/common/physics.hpp:130-138).
__device__ double phase_count(const double *tab, int Ls, int L, int wave, double c) {
  const double ic = 1. / (c * c);
  double n = 0.;
  for (int j = 0; j < L - 1; ++j) {
    const double h = tab[j];
    if (h == 0.) continue;
    const double ivs = tab[2 * Ls + j], ivp = tab[Ls + j];
    const double zs = ivs * ivs - ic;
    if (zs > 0.) n += h * sqrt(zs);
    if (!wave) {
      const double zp = ivp * ivp - ic;
      if (zp > 0.) n += h * sqrt(zp);
    }
  }
  return 2. * n;
}

// ---------------------------------------------------------------------------
// prep_models: one warp per model.
// Shared memory per warp: 2 * sortcap doubles + 2 * sortcap ints.
// ---------------------------------------------------------------------------
__global__ void prep_models(Dev d, int sortcap, int automatic) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int b = blockIdx.x * (blockDim.x >> 5) + wib;
  if (b >= d.B) return;
  double *skey = reinterpret_cast<double *>(smem_raw) + static_cast<size_t>(wib) * sortcap;
  int *sval = reinterpret_cast<int *>(reinterpret_cast<double *>(smem_raw) +
                                      static_cast<size_t>(blockDim.x >> 5) * sortcap) +
              static_cast<size_t>(wib) * sortcap;
  const int Lmax = d.Lmax, Ls = d.Ls;
  const size_t in = static_cast<size_t>(b) * Lmax;
  double *t64 = d.layer64 + static_cast<size_t>(b) * ROWS * Ls;
  float *t32 = d.layer32 + static_cast<size_t>(b) * ROWS * Ls;

  // 1. keep row 0, the half-space and every layer of positive thickness; a
  //    zero-thickness layer is an identity step of the recurrence.
  int L = 0;
  for (int base = 0; base < Lmax; base += 32) {
    const int j = base + lane;
    bool keep = false;
    double hj = 0., vpj = 1., vsj = 0., rj = 1.;
    if (j < Lmax) {
      hj = d.h[in + j];
      vpj = d.vp[in + j];
      vsj = d.vs[in + j];
      rj = d.rho[in + j];
      keep = j == 0 || j == Lmax - 1 || hj > 0.;
    }
    const unsigned mask = __ballot_sync(FULL, keep);
    if (keep) {
      const int r = L + __popc(mask & lanemask_lt());
      const double ivp = 1. / vpj, ivs = vsj > 0. ? 1. / vsj : 0.;
      const double vals[ROWS] = {j == Lmax - 1 ? 0. : hj, ivp, ivs, vsj * vsj, rj, 1. / rj,
                                 vsj > 0. ? 1. / (rj * vsj * vsj) : 0., vpj, vsj};
#pragma unroll
      for (int q = 0; q < ROWS; ++q) {
        t64[q * Ls + r] = vals[q];
        t32[q * Ls + r] = static_cast<float>(vals[q]);
      }
    }
    L += __popc(mask);
  }
  __syncwarp();
  const double *vpr = t64 + 7 * Ls, *vsr = t64 + 8 * Ls, *hr = t64, *rr = t64 + 4 * Ls;
  const int water = vsr[0] == 0. ? 1 : 0;
  const int top = water;
  const int wave = d.wave;

  // 2. search window (cpp/cpu/solver.cpp:781-790, cpp/common/physics.hpp:158-175).
  //    A given window is used as is, except that a non-positive lower bound asks
  //    for the automatic one and the upper bound never exceeds the half-space
  //    shear velocity (exclusive).
  double lo = d.bounds_in ? d.bounds_in[2 * b] : 0.;
  double hi = d.bounds_in ? d.bounds_in[2 * b + 1] : INFINITY;
  if (automatic || !(lo > 0.)) {
    double best = 1e300;
    for (int j = top + lane; j < L; j += 32) {
      if (hr[j] == 0. && j < L - 1) continue;  // a zero-thickness row carries no waves
      const double s = vsr[j], p = vpr[j];
      double x = wave ? s : rayleigh_speed(p, s);
      if (!wave && top) x = fmin(x, scholte_speed(vpr[0], rr[0], p, s, rr[j]));
      best = fmin(best, x);
    }
    for (int o = 16; o; o >>= 1) best = fmin(best, __shfl_xor_sync(FULL, best, o));
    lo = .125 * best;
  }
  hi = fmin(hi, nextafter(vsr[L - 1], 0.));
  int state = hi > lo ? 0 : -4;
  if (state == 0 && wave) {  // SH guide: a finite layer slower than the half-space
    bool guide = false;
    for (int j = top + lane; j < L - 1; j += 32) guide |= hr[j] > 0. && vsr[j] < vsr[L - 1];
    if (!__any_sync(FULL, guide)) state = -3;
  }
  if (lane == 0) {
    d.mL[b] = L;
    d.mwater[b] = water;
    d.mstate[b] = state;
    d.mlo[b] = lo;
    d.mhi[b] = hi;
    d.mtail[2 * b] = hi;
    d.mtail[2 * b + 1] = vsr[L - 1] * (1. + -1 * 1e-7);  // the -1e-7 seed of the half-space row
    if (d.bounds_out) {
      d.bounds_out[2 * b] = lo;
      d.bounds_out[2 * b + 1] = hi;
    }
  }
  if (state) return;

  // 3. knot table: log-spaced points over [lo, hi] plus every finite-layer body
  //    velocity inside the window (kinks of N(c)), sorted.
  const int nlog = d.nlog;
  const double lspan = log(hi / lo);
  int n = 0;
  for (int i = lane; i <= nlog; i += 32) {
    skey[i] = i == 0 ? lo : (i == nlog ? hi : lo * exp(lspan * i / nlog));
    sval[i] = 0;
  }
  n = nlog + 1;
  for (int base = top; base < L - 1; base += 32) {
    const int j = base + lane;
    bool ks = false, kp = false;
    double s = 0., p = 0.;
    if (j < L - 1 && hr[j] > 0.) {
      s = vsr[j];
      p = vpr[j];
      ks = s > lo && s < hi;
      kp = !wave && p > lo && p < hi;
    }
    const unsigned ms = __ballot_sync(FULL, ks), mp = __ballot_sync(FULL, kp);
    if (ks) {
      const int r = n + __popc(ms & lanemask_lt());
      skey[r] = s;
      sval[r] = 1;
    }
    n += __popc(ms);
    if (kp) {
      const int r = n + __popc(mp & lanemask_lt());
      skey[r] = p;
      sval[r] = 1;
    }
    n += __popc(mp);
  }
  int n2 = pow2_ceil(n);
  for (int i = n + lane; i < n2; i += 32) {
    skey[i] = INFINITY;
    sval[i] = 0;
  }
  __syncwarp();
  warp_bitonic(skey, sval, n2, lane);
  // Keep the last element of each run of equal keys, merging kink marks.
  int nk = 0;
  double4 *kt = d.knot + static_cast<size_t>(b) * d.nkmax;
  for (int base = 0; base < n; base += 32) {
    const int i = base + lane;
    bool keep = false;
    double c = 0.;
    int kink = 0;
    if (i < n) {
      c = skey[i];
      keep = i + 1 >= n || skey[i + 1] != c;
      kink = sval[i] | (i > 0 && skey[i - 1] == c ? sval[i - 1] : 0);
    }
    const unsigned mask = __ballot_sync(FULL, keep);
    if (keep) {
      const int r = nk + __popc(mask & lanemask_lt());
      kt[r] = make_double4(c, 0., log(c), kink ? 1. : 0.);
    }
    nk += __popc(mask);
  }
  __syncwarp();
  // N(c) at each knot, and the kink term of the interval starting at a kink.
  for (int i = lane; i < nk; i += 32) {
    double4 q = kt[i];
    q.y = phase_count(t64, Ls, L, wave, q.x);
    double kink = 0.;
    if (q.w != 0. && i + 1 < nk) {
      const double c1 = kt[i + 1].x, ic1 = 1. / (c1 * c1);
      for (int j = top; j < L - 1; ++j) {
        if (hr[j] == 0.) continue;
        if (vsr[j] == q.x) kink += hr[j] * sqrt(fmax(0., 1. / (vsr[j] * vsr[j]) - ic1));
        if (!wave && vpr[j] == q.x) kink += hr[j] * sqrt(fmax(0., 1. / (vpr[j] * vpr[j]) - ic1));
      }
    }
    q.w = 2. * kink;
    kt[i] = q;
  }
  __syncwarp();
  if (lane == 0) {
    d.nknot[b] = nk;
    // log weight: background spacing ln(hi/lo)/log_points in ln c per scan step
    d.malpha[b] = static_cast<double>(nlog) / (d.density * lspan);
  }

  // 4. seed points: the window ends, every body velocity and its +-1e-7 neighbours,
  //    the top-layer Rayleigh/Love and Scholte speeds with nearby offsets
  //    (the sampling seeds of cpp/cpu/solver.cpp:482-495).
  __syncwarp();
  n = 0;
  const int seed_top = wave && water ? 1 : 0;
  for (int base = seed_top; base < L; base += 32) {
    const int j = base + lane;
    double v[6];
    int cnt = 0;
    if (j < L) {
      const double vv[2] = {vpr[j], vsr[j]};
      for (int q = 0; q < 2; ++q)
        for (int side = -1; side <= 1; ++side) {
          const double c = vv[q] * (1. + side * 1e-7);
          if (c > lo && c < hi) v[cnt++] = c;
        }
    }
    int off = cnt;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(FULL, off, o);
      if (lane >= o) off += y;
    }
    const int total = __shfl_sync(FULL, off, 31);
    off -= cnt;
    for (int q = 0; q < cnt; ++q) {
      skey[n + off + q] = v[q];
      sval[n + off + q] = 0;
    }
    n += total;
  }
  __syncwarp();
  if (lane == 0) {
    const double s0 = wave ? vsr[top] : rayleigh_speed(vpr[top], vsr[top]);
    const double ws = (!wave && top) ? scholte_speed(vpr[0], rr[0], vpr[1], vsr[1], rr[1]) : NAN;
    const double gaps[5] = {1e-7, 1e-6, 1e-5, 1e-4, 1e-3};
    const double base[2] = {s0, ws};
    skey[n++] = lo;
    skey[n++] = hi;
    for (int q = 0; q < 2; ++q) {
      const double s = base[q];
      const double cands[2] = {s, .9 * s};
      for (int r = 0; r < 2; ++r)
        if (cands[r] > lo && cands[r] < hi) skey[n++] = cands[r];
      for (int g = 0; g < 5; ++g) {
        const double a = s * (1. - gaps[g]), c = s * (1. + gaps[g]);
        if (a > lo && a < hi) skey[n++] = a;
        if (c > lo && c < hi) skey[n++] = c;
      }
    }
  }
  n = __shfl_sync(FULL, n, 0);
  __syncwarp();
  n2 = pow2_ceil(n);
  for (int i = n + lane; i < n2; i += 32) skey[i] = INFINITY;
  for (int i = lane; i < n2; i += 32) sval[i] = 0;
  __syncwarp();
  warp_bitonic(skey, sval, n2, lane);
  int ns = 0;
  double *sd = d.seed + static_cast<size_t>(b) * d.nsmax;
  for (int base = 0; base < n; base += 32) {
    const int i = base + lane;
    const bool keep = i < n && (i == 0 || skey[i - 1] != skey[i]);
    const unsigned mask = __ballot_sync(FULL, keep);
    if (keep) sd[ns + __popc(mask & lanemask_lt())] = skey[i];
    ns += __popc(mask);
  }
  if (lane == 0) d.nseed[b] = ns;
}

// ---------------------------------------------------------------------------
// init_traces: the round-0 trace list (period-major) and per-trace resets;
// with anchor continuation, targets go to their own list.
// ---------------------------------------------------------------------------
__global__ void init_traces(Dev d) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= d.n_traces) return;
  int b, t, role = 0;  // role: 1 continuation anchor, 2 continuation target
  if (d.ragged) {
    // CSR order; the owning model by binary search of the offsets
    t = q;
    int lo = 0, hi = d.B;  // r_offsets[lo] <= t < r_offsets[hi]
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (d.r_offsets[mid] <= t) lo = mid;
      else hi = mid;
    }
    b = lo;
    const int f = t - d.r_offsets[b];
    d.tr_model[t] = b;
    d.tr_period[t] = d.periods[t];
    d.tr_out[t] = d.r_outbase[b] + f;
    d.tr_stride[t] = d.r_offsets[b + 1] - d.r_offsets[b];
    const int mb = d.r_modes[b];
    d.tr_modes[t] = mb < 1 ? 1 : (mb > d.nmodes ? d.nmodes : mb);  // the bracket slots hold nmodes + 2
  } else {
    b = q % d.B;
    const int f = q / d.B;
    t = b * d.T + f;
    d.tr_model[t] = b;
    d.tr_period[t] = d.periods[f];
    d.tr_out[t] = static_cast<long long>(b) * d.nmodes * d.T + f;
    d.tr_stride[t] = d.T;
    d.tr_modes[t] = d.nmodes;
  }
  if (d.crole) role = d.crole[t];
  d.nbr[t] = 0;
  d.tflags[t] = 0;
  // PredictionFlag: ANCHOR (1), a target's verdict later, else searched
  // independently (BYPASSED, 8)
  if (d.pred) d.pred[t] = role == 1 ? 1u : (role == 2 && d.mstate[b] == 0 ? 0u : 8u);
  if (d.mstate[b] == 0) {
    if (role == 2) {
      const int pos = atomicAdd(&d.ctr[C_NTARGET], 1);
      d.cont_list[pos] = t;
    } else {
      const int pos = atomicAdd(&d.ctr[C_NTRACE], 1);
      d.trace_list[pos] = t;
    }
  }
}

// FP64 values at the two near-cutoff positions of every trace, for the FP32
// scan (one thread per trace, all lanes busy): near the half-space cutoff the
// start vector depends on the small radical sqrt(k^2 - kb^2) directly, which
// single precision resolves poorly.
__global__ void tail_values(Dev d) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= *(volatile int *)&d.ctr[C_NTRACE]) return;
  const int t = d.trace_list[q];
  const int b = d.tr_model[t];
  const double w = TWO_PI / d.tr_period[t];
  const LayerView<double> m = make_view<double>(d.layer64 + static_cast<size_t>(b) * ROWS * d.Ls, d.Ls,
                                                d.mL[b], d.mwater[b]);
  for (int i = 0; i < 2; ++i) {
    const double c = d.mtail[2 * b + i];
    double g = 0., lm = 0., F = NAN;
    if (c > d.mlo[b]) F = secular<double, double>(m, d.wave, w / c, w, &g, &lm);
    d.tail[2 * static_cast<size_t>(t) + i] = make_double4(c, F, g, lm);
  }
}

// Position of scan point j (1 <= j <= J) of a trace: invert
// u(c) = f N(c) + alpha ln c at u_lo + j / density through the knot table.  In
// an interval that starts at a body velocity the kink term grows like
// sqrt(c - c_i); the local model u = u_i + a sqrt(s) + b s (s the fractional
// position) is inverted exactly.
//
// `from` is a knot index at or below the interval of `target` (each lane's
// targets increase from step to step, so the lane's previous interval
// qualifies): the interval is found by galloping up from it and bisecting the
// last gap -- the same interval a bisection of the whole table finds (the last
// knot with u <= target), in a few table reads instead of ~8 dependent ones.
// On return `from` holds that interval.
__device__ __forceinline__ double scan_point(const double4 *kt, int nk, double f, double alpha, double target,
                                             int &from) {
  int lo = from, hi = nk - 1;
  for (int gap = 1; lo + gap < hi; gap <<= 1) {
    const double4 q = kt[lo + gap];
    if (fma(f, q.y, alpha * q.z) <= target) lo += gap;
    else {
      hi = lo + gap;
      break;
    }
  }
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    const double4 q = kt[mid];
    if (fma(f, q.y, alpha * q.z) <= target) lo = mid; else hi = mid;
  }
  from = lo;
  const double4 q0 = kt[lo], q1 = kt[hi];
  const double u0 = fma(f, q0.y, alpha * q0.z), u1 = fma(f, q1.y, alpha * q1.z);
  // the fractional position within the knot interval needs only single precision
  const float dt = static_cast<float>(fmax(0., target - u0)), du = static_cast<float>(u1 - u0);
  const float a = static_cast<float>(f * q0.w), bs = fmaxf(0.f, du - a);
  float s = 0.f;
  if (du > 0.f && dt > 0.f) {  // (dt = 0 would give 0/0 where the interval has no kink)
    const float x = 2.f * dt / (a + sqrtf(a * a + 4.f * bs * dt));
    s = fminf(1.f, x * x);
  }
  return fma(q1.x - q0.x, static_cast<double>(s), q0.x);
}

// Index (0..32) of the first lane whose sorted value is >= x (or > x when
// `inclusive`), over the warp's ascending per-lane values `v`.
__device__ __forceinline__ int warp_rank(double v, double x, bool inclusive) {
  int lo = 0, hi = 32;
#pragma unroll
  for (int it = 0; it < 6; ++it) {
    const int mid = (lo + hi) >> 1;
    const double m = __shfl_sync(FULL, v, mid & 31);
    const bool less = inclusive ? (m <= x) : (m < x);
    if (lo < hi) {
      if (less) lo = mid + 1; else hi = mid;
    }
  }
  return lo;
}

// Global-memory FP64 view of model b.
__device__ __forceinline__ LayerView<double> global_view(const Dev &d, int b) {
  return make_view<double>(layer_table<double>(d, b), d.Ls, d.mL[b], d.mwater[b]);
}

// Append one bracket to slot r of a trace (flo/fhi NaN: unknown in FP64).
__device__ __forceinline__ void put_bracket(double *slot, int r, double lo, double hi, double flo,
                                            double fhi) {
  double *s = slot + static_cast<size_t>(r) * SLOT;
  s[0] = lo;
  s[1] = hi;
  s[2] = flo;
  s[3] = fhi;
  s[4] = NAN;
}

// Could a same-sign local minimum (v at x1, neighbours u at x0 and z at x2, all
// of one sign, s*g > 0) hide a root pair?  Close pairs show up in the shape
// feature as a V whose flanks are nearly linear and whose bottom dips through
// zero between samples; a smooth minimum well above zero does not.  The trough
// is kept when a V with its vertex on zero fits the samples -- the linear
// extension of either flank reaches zero before the far neighbour -- or when a
// parabola through the three samples dips to zero.
// `noise_l` and `noise_r` are the rounding noise of the left (u, v) and right
// (v, z) sample pairs.
__device__ __forceinline__ bool trough_may_hide_roots(double x0, double x1, double x2, float u, float v, float z,
                                                      float noise_l = 1e-7f, float noise_r = 1e-7f) {
  // both flanks must rise by more than the evaluations' rounding noise
  if (!(v + noise_l < u && v + noise_r < z) || !(x0 < x1 && x1 < x2)) return false;
  // single precision suffices for the slope test: spacings are differences of
  // exact positions, well above float resolution
  const float h0 = static_cast<float>(x1 - x0), h1 = static_cast<float>(x2 - x1);
  const float sl = (u - v) / h0, sr = (z - v) / h1;  // flank steepness (> 0)
  if (v / sl < 1.25f * h1 || v / sr < 1.25f * h0) return true;
  const float d1 = -sl, d2 = sr, a2 = (d2 - d1) / (h0 + h1);
  if (a2 > 0.f) {
    const float xs = .5f * h0 - d1 / (2.f * a2);  // vertex offset from x0
    if (u + d1 * xs + a2 * xs * (xs - h0) <= 0.f) return true;
  }
  return false;
}

// Depth (base-2 log units) of the middle sample's log-magnitude below the chord
// of its neighbours: large where the whole unnormalised vector nearly vanishes,
// which hides a root pair even where the shape feature stays smooth.
constexpr double MDIP = 0.5;
__device__ __forceinline__ float magnitude_dip(double x0, double x1, double x2, float m0, float m1, float m2) {
  if (!(x0 < x1 && x1 < x2) || !(m1 < m0 && m1 < m2)) return 0.f;
  const float t = static_cast<float>((x1 - x0) / (x2 - x0));
  return m0 + t * (m2 - m0) - m1;
}

// Warp-cooperative FP64 zoom into a same-sign trough of the shape feature:
// 32 points inside (a, b) per step; a sign change among them yields brackets
// (appended in order, FP64 values known); otherwise the window shrinks 16.5x
// around the smallest s*g until the minimum is resolved above zero or the
// window reaches the refinement width.  `sa`, `sb` are s*g at a and b.
template <int WAVE>
__device__ __noinline__ int zoom_trough(const LayerView<double> &m, double w, double a, double b,
                                       double sa, double sb, double ma, double mb, double sgn, int mode,
                                       double tol, double *slot, int nbr, int K, int lane,
                                       unsigned long long &evals) {
  const bool neg = sgn < 0.;
  double Fa = NAN, Fb = NAN;  // FP64 values of the window ends once they are zoom points
  for (int it = 0; it < 10; ++it) {
    const double width = b - a;
    if (!(width > fmax(4e-15 * b, .125 * tol * b))) break;
    const double x = a + width * (lane + 1) * (1. / 33.);
    double g, lm;
    const double F = secular<double, double>(m, WAVE, w / x, w, &g, &lm);
    evals += 32;
    const bool opp = signbit(F) != neg;
    const unsigned om = __ballot_sync(FULL, opp);
    if (om) {
      // brackets between consecutive points of a, x_0..x_31, b (a and b have sign sgn)
      const double xl = __shfl_up_sync(FULL, x, 1), Fl = __shfl_up_sync(FULL, F, 1);
      const bool opl = lane ? ((om >> (lane - 1)) & 1) != 0 : false;
      const bool left = opp != opl;                    // change between element lane-1 (or a) and lane
      const bool right = lane == 31 && opp;            // change between x_31 and b
      const unsigned lm_ = __ballot_sync(FULL, left), rm = __ballot_sync(FULL, right);
      if (left) {
        const int r = nbr + __popc(lm_ & lanemask_lt());
        if (r < K) put_bracket(slot, r, lane ? xl : a, x, lane ? Fl : Fa, F);
      }
      nbr += __popc(lm_);
      if (right) {
        if (nbr < K) put_bracket(slot, nbr, x, b, F, Fb);
      }
      nbr += __popc(rm);
      return nbr < K ? nbr : K;
    }
    // no sign change: zoom on the lowest s*g (mode 0) or log-magnitude (mode 1)
    const double v = sgn * g;
    const double key = mode ? lm : v;
    double best = key;
    int arg = lane;
    for (int o = 16; o; o >>= 1) {
      const double ob = __shfl_xor_sync(FULL, best, o);
      const int oa = __shfl_xor_sync(FULL, arg, o);
      if (ob < best || (ob == best && oa < arg)) { best = ob; arg = oa; }
    }
    const int il = (arg - 1) & 31, ir = (arg + 1) & 31;
    const double vl = arg ? __shfl_sync(FULL, v, il) : sa;
    const double vr = arg < 31 ? __shfl_sync(FULL, v, ir) : sb;
    const double ml = arg ? __shfl_sync(FULL, lm, il) : ma;
    const double mr = arg < 31 ? __shfl_sync(FULL, lm, ir) : mb;
    const double xlo = arg ? __shfl_sync(FULL, x, il) : a;
    const double xhi = arg < 31 ? __shfl_sync(FULL, x, ir) : b;
    const double Flo = arg ? __shfl_sync(FULL, F, il) : Fa;
    const double Fhi = arg < 31 ? __shfl_sync(FULL, F, ir) : Fb;
    const double xm = __shfl_sync(FULL, x, arg);
    // stop once the lowest sample and its neighbours no longer admit a hidden pair
    const bool go = mode ? magnitude_dip(xlo, xm, xhi, ml, __shfl_sync(FULL, lm, arg), mr) > MDIP
                         : trough_may_hide_roots(xlo, xm, xhi, vl, __shfl_sync(FULL, v, arg), vr);
    if (!go) break;
    a = xlo; b = xhi; sa = vl; sb = vr; ma = ml; mb = mr; Fa = Flo; Fb = Fhi;
  }
  return nbr;
}

// Shape-feature magnitude below which a single-precision sample's sign is not
// trusted: the sample is evaluated again in FP64.
#ifndef MD200_REDO_G
#define MD200_REDO_G 2e-4
#endif

// Single-precision screen of a trough window, run before the FP64 zoom in the
// FP32 scan: up to two 32-point steps in FP32 (the model table in shared
// memory).  Returns true when the window is dismissed -- no sample changes sign
// or comes near zero (|g| <= 2e-4), and the lowest sample no longer admits a
// hidden pair -- so only troughs that stay suspicious pay for FP64.
template <int WAVE>
__device__ __noinline__ bool screen_trough32(const LayerView<float> &m, float w, double a, double b, double sa,
                                             double sb, double ma, double mb, double sgn, int mode, int lane,
                                             unsigned long long &evals) {
  const bool neg = sgn < 0.;
  for (int it = 0; it < 2; ++it) {
    const double width = b - a;
    if (!(width > 1e-5 * b)) return false;  // below single-precision resolution
    const double x = a + width * (lane + 1) * (1. / 33.);
    const float x32 = static_cast<float>(x);
    float g, lm;
    const float F = secular<float, float>(m, WAVE, w / x32, w, &g, &lm);
    evals += 32;
    const bool doubt = signbit(F) != neg || !(fabsf(g) > static_cast<float>(MD200_REDO_G)) || !isfinite(F);
    if (__any_sync(FULL, doubt)) return false;
    const double v = sgn * g;
    const double key = mode ? lm : v;
    double best = key;
    int arg = lane;
    for (int o = 16; o; o >>= 1) {
      const double ob = __shfl_xor_sync(FULL, best, o);
      const int oa = __shfl_xor_sync(FULL, arg, o);
      if (ob < best || (ob == best && oa < arg)) { best = ob; arg = oa; }
    }
    const int il = (arg - 1) & 31, ir = (arg + 1) & 31;
    const double vl = arg ? __shfl_sync(FULL, v, il) : sa, vr = arg < 31 ? __shfl_sync(FULL, v, ir) : sb;
    const double ml = arg ? __shfl_sync(FULL, static_cast<double>(lm), il) : ma;
    const double mr = arg < 31 ? __shfl_sync(FULL, static_cast<double>(lm), ir) : mb;
    const double xlo = arg ? __shfl_sync(FULL, x, il) : a, xhi = arg < 31 ? __shfl_sync(FULL, x, ir) : b;
    const double xm = __shfl_sync(FULL, x, arg);
    const bool go = mode ? magnitude_dip(xlo, xm, xhi, ml, __shfl_sync(FULL, static_cast<double>(lm), arg), mr) > MDIP
                         : trough_may_hide_roots(xlo, xm, xhi, vl, __shfl_sync(FULL, v, arg), vr, 1e-5f, 1e-5f);
    if (!go) return true;
    a = xlo; b = xhi; sa = vl; sb = vr; ma = ml; mb = mr;
  }
  return false;
}

// ---------------------------------------------------------------------------
// scan<T, WAVE>: persistent, one warp per trace.
// Shared memory per warp: EVAL_ROWS * Ls values of T (model table) + 32 doubles
// (merge buffer).
//
// Trough tests look only at "regular" samples -- a sample within 1e-6 of its
// left neighbour (the +-1e-7 seeds that straddle a body velocity, where the
// shape feature has a square-root kink) takes part in sign-change bracketing
// but not in slope estimates -- and a trough window must lie inside one sign
// segment (no sign change anywhere between its ends), so a zoom never revisits
// a root the brackets already hold.
// ---------------------------------------------------------------------------
// A sample as the trough tests see it: position, shape feature and log-magnitude
// (single precision suffices for slopes and dips), sign segment and sign.
struct Sample {
  double c;
  float g, M;
  int seg;  // running sign-change count; bit 29: value evaluated in FP64; bit 30: sign of F
};

__device__ __forceinline__ Sample shfl_sample(const Sample &s, int src) {
  Sample r;
  r.c = __shfl_sync(FULL, s.c, src);
  r.g = __shfl_sync(FULL, s.g, src);
  r.M = __shfl_sync(FULL, s.M, src);
  r.seg = __shfl_sync(FULL, s.seg, src);
  return r;
}
__device__ __forceinline__ double sample_sign(const Sample &s) { return (s.seg >> 30) & 1 ? -1. : 1.; }
__device__ __forceinline__ int sample_segment(const Sample &s) { return s.seg & 0x1fffffff; }
__device__ __forceinline__ bool sample_exact(const Sample &s) { return (s.seg >> 29) & 1; }
// Rounding noise of the shape-feature difference of two samples: single
// precision unless both were evaluated in FP64 (the sign-uncertain samples of the
// FP32 scan are, so troughs whose floor lies in that band keep the FP64 test).
__device__ __forceinline__ float pair_noise(bool single, const Sample &a, const Sample &b) {
  return single && !(sample_exact(a) && sample_exact(b)) ? 1e-5f : 1e-7f;
}

// The last cell of a window: its right end is the window end, which no V test
// sees as a middle sample.  When the shape feature falls into the end steeply
// enough that its linear extension would reach zero within one more cell (the
// left-flank test of trough_may_hide_roots, mirrored), a pair may hide in the
// cell: it is screened and zoomed like an interior trough.  R2, R1: the last two
// regular samples, in one sign segment.  Out of line: it runs once per trace,
// after the scan loop, and keeps its registers out of the loop's allocation.
template <class T, int WAVE>
__device__ __noinline__ int last_cell(const LayerView<T> view, const LayerView<double> view64, double w, Sample R2,
                                      Sample R1, double tol, double *slot, int nbr, int K, int lane, int nsteps,
                                      unsigned long long &evals, unsigned long long &evals32,
                                      unsigned long long &steps, unsigned long long &steps32,
                                      unsigned long long &zooms) {
  constexpr bool single = sizeof(T) == 4;
  const double sgn = sample_sign(R1);
  const float u = static_cast<float>(sgn) * R2.g, v = static_cast<float>(sgn) * R1.g;
  const float h0 = static_cast<float>(R1.c - R2.c);
  const float noise = pair_noise(single, R2, R1);
  if (!(u > v + noise && v / ((u - v) / h0) < 1.25f * h0)) return nbr;
  bool dismissed = false;
  if constexpr (single) {
    unsigned long long se = 0;
    dismissed = screen_trough32<WAVE>(view, static_cast<float>(w), R2.c, R1.c, u, v, R2.M, R1.M, sgn, 0, lane, se);
    evals += se;
    evals32 += se;
    steps += se * nsteps;
    steps32 += se * nsteps;
  }
  if (!dismissed) {
    unsigned long long ze = 0;
    nbr = zoom_trough<WAVE>(view64, w, R2.c, R1.c, u, v, R2.M, R1.M, sgn, 0, tol, slot, nbr, K, lane, ze);
    evals += ze;
    steps += ze * nsteps;
    ++zooms;
  }
  return nbr;
}

#ifndef MD200_SCAN_MIN_BLOCKS
#define MD200_SCAN_MIN_BLOCKS 4
#endif
// resident CTAs per SM the single-precision Love scan is compiled for (its
// recurrence is a 2-vector: fewer live registers than the Rayleigh scan's)
#ifndef MD200_SCAN_MIN_BLOCKS_LOVE32
#define MD200_SCAN_MIN_BLOCKS_LOVE32 MD200_SCAN_MIN_BLOCKS
#endif

// ---------------------------------------------------------------------------
// The scan of one trace as a sequence of 32-sample steps: positions, values,
// bookkeeping.  One warp runs a trace from start to end (persistent kernel
// `scan`, the model table in shared memory).  The same steps also run as rounds
// of separate kernels over an active set of traces (split_scan.cuh), with the
// state below carried in global memory between rounds; the fused kernel then
// finishes, in resume mode, the traces the rounds left unfinished.
// ---------------------------------------------------------------------------

// Per-trace scan state carried between steps.
struct ScanState {
  long long gi, J;         // next grid index, last grid index
  int si, nbr, nseg;       // next seed, brackets held, sign changes so far
  unsigned tfl;            // trace flags
  int bits;                // 1 have1, 2 hr1, 4 hr2, 8 ex1, 16 finished
  double c1, F1;           // the last sample (bracketing against the next step)
  double zoom_right;       // right end of the last zoomed window (windows never overlap)
  Sample R1, R2;           // the last two regular samples
};
constexpr int SS_HAVE1 = 1, SS_HR1 = 2, SS_HR2 = 4, SS_EX1 = 8, SS_FINISHED = 16;

// Trace constants (recomputed wherever a trace is picked up).
struct TraceCtx {
  int t, b, K, nsteps, nk, ns;
  double w, fr, alpha, u_lo, hi;
  const double4 *kt;
  const double *sd;
  double *slot;
  const double4 *tail;
};

struct ScanCounters {
  unsigned long long evals = 0, evals32 = 0, steps = 0, steps32 = 0, zooms = 0;
};

__device__ __forceinline__ TraceCtx trace_ctx(const Dev &d, int t) {
  TraceCtx x;
  x.t = t;
  x.b = d.tr_model[t];
  x.K = d.tr_modes[t] + 2;  // nmodes + 2 guard roots
  const double period = d.tr_period[t];
  x.w = TWO_PI / period;
  x.fr = 1. / period;
  x.nsteps = layer_steps(d.mL[x.b], d.mwater[x.b]);
  x.kt = d.knot + static_cast<size_t>(x.b) * d.nkmax;
  x.nk = d.nknot[x.b];
  x.alpha = d.malpha[x.b];
  x.u_lo = fma(x.fr, x.kt[0].y, x.alpha * x.kt[0].z);
  x.sd = d.seed + static_cast<size_t>(x.b) * d.nsmax;
  x.ns = d.nseed[x.b];
  x.hi = d.mhi[x.b];
  x.slot = d.slot + static_cast<size_t>(t) * d.KB * SLOT;
  x.tail = d.tail + 2 * static_cast<size_t>(t);
  return x;
}

__device__ __forceinline__ ScanState scan_start(const Dev &d, const TraceCtx &x) {
  ScanState st;
  const double u_hi = fma(x.fr, x.kt[x.nk - 1].y, x.alpha * x.kt[x.nk - 1].z);
  long long J = static_cast<long long>(ceil((u_hi - x.u_lo) * d.density)) - 1;
  st.tfl = 0;
  if (J < 0) J = 0;
  if (J > d.jmax) {
    J = d.jmax;
    st.tfl |= TRACE_WORKSPACE_LIMIT;
  }
  st.J = J;
  st.gi = 1;
  st.si = st.nbr = st.nseg = 0;
  st.bits = 0;
  st.c1 = st.F1 = 0.;
  st.zoom_right = -INFINITY;
  st.R1 = Sample{0., 0.f, 0.f, 0};
  st.R2 = Sample{0., 0.f, 0.f, 0};
  return st;
}

// The next 32 sample positions: grid points and seeds merged in order (this
// lane's position in c; INFINITY past the window).  Returns the valid-lane mask;
// with SRC, also (*seeds) the lanes whose position is a seed (kbuf: 32 bytes of
// shared memory beside mbuf).
template <bool SRC = false>
__device__ __forceinline__ unsigned scan_positions(const TraceCtx &x, ScanState &st, double step, int lane,
                                                   double *mbuf, int &kfrom, double &c,
                                                   unsigned char *kbuf = nullptr, unsigned *seeds = nullptr) {
  const long long gj = st.gi + lane;
  const double gv = gj <= st.J ? scan_point(x.kt, x.nk, x.fr, x.alpha, x.u_lo + static_cast<double>(gj) * step,
                                            kfrom)
                               : INFINITY;
  double sv = st.si + lane < x.ns ? x.sd[st.si + lane] : INFINITY;
  if ((st.tfl & TRACE_WORKSPACE_LIMIT) && st.gi + 31 >= st.J) {
    // a capped grid ends in this step (or has ended): seeds past its last point
    // lie outside the first search -- between seeds alone, roots would be
    // skipped -- so the scan stops there and the trace goes to the fallback
    double last = gj <= st.J ? gv : -INFINITY;
    for (int o = 16; o; o >>= 1) last = fmax(last, __shfl_xor_sync(FULL, last, o));
    if (sv > last) sv = INFINITY;
  }
  // a step of grid points only: 32 finite grid points and the next seed at or
  // above the last of them, so the merge would keep the grid points in place
  const double g31 = __shfl_sync(FULL, gv, 31), s0 = __shfl_sync(FULL, sv, 0);
  if (g31 < INFINITY && s0 >= g31) {
    c = gv;
    if constexpr (SRC) *seeds = 0u;
    st.gi += 32;
    return FULL;
  }
  const int rg = warp_rank(sv, gv, false);  // seeds strictly below this scan point
  const int rs = warp_rank(gv, sv, true);   // scan points at or below this seed
  const int pg = lane + rg, ps = lane + rs;
  mbuf[lane] = INFINITY;
  __syncwarp();
  if (pg < 32) mbuf[pg] = gv;
  if (ps < 32) mbuf[ps] = sv;
  if constexpr (SRC) {
    if (pg < 32) kbuf[pg] = 0;
    if (ps < 32) kbuf[ps] = 1;
  }
  __syncwarp();
  c = mbuf[lane];
  if constexpr (SRC) *seeds = __ballot_sync(FULL, c < INFINITY && kbuf[lane]);
  __syncwarp();
  st.gi += __popc(__ballot_sync(FULL, pg < 32 && gv < INFINITY));
  st.si += __popc(__ballot_sync(FULL, ps < 32 && sv < INFINITY));
  return __ballot_sync(FULL, c < INFINITY);
}

// Single-precision position of a sample (FP32 scan): rounded to float and kept
// below hi, except in the near-cutoff band, whose samples stay at their exact
// positions and are evaluated in FP64 only.
__device__ __forceinline__ float scan_position32(double &c, double hi, bool &near_cut) {
  const bool valid = c < INFINITY;
  near_cut = valid && c >= hi * (1. - 1e-4);
  float x = valid ? static_cast<float>(c) : 1.f;
  if (valid && static_cast<double>(x) > hi) x = nextafterf(x, 0.f);
  if (valid && !near_cut) c = static_cast<double>(x);
  return x;
}

// FP64 completion of a single-precision sample: the near-cutoff band takes the
// trace's precomputed FP64 values where they match, and sign-uncertain samples
// (small |g|) and the rest of that band are evaluated in FP64.  Returns true
// when this lane needed an FP64 evaluation.
template <int WAVE>
__device__ __forceinline__ bool scan_complete32(const LayerView<double> &view64, double w, const double4 *tail,
                                                double c, bool valid, bool near_cut, double &F, double &g, double &M,
                                                bool &exact) {
  bool have_tail = false;
  exact = false;
  if (near_cut) {
    const double4 t0 = tail[0], t1 = tail[1];
    const double4 tv = c == t0.x ? t0 : t1;
    if (c == tv.x && isfinite(tv.y)) {
      F = tv.y;
      g = tv.z;
      M = tv.w;
      exact = true;
      have_tail = true;
    }
  }
  const bool redo = valid && !have_tail && (!(fabs(g) > MD200_REDO_G) || near_cut);
  if (redo) {
    F = eval64_outline(view64, WAVE, w, c, &g, &M);
    exact = true;
  }
  return redo;
}

// One step's bookkeeping: brackets from sign changes, trough tests and zooms,
// the carries.  `vm`: valid lanes of the step.
template <class T, int WAVE>
__device__ __forceinline__ void scan_bookkeep(const Dev &d, const TraceCtx &x, ScanState &st, const LayerView<T> &view,
                                              const LayerView<double> &view64, int lane, double c, double F,
                                              double g, double M, bool exact, unsigned vm, ScanCounters &ctr) {
  constexpr bool single = sizeof(T) == 4;
  const unsigned lt = lanemask_lt(), le = lt | (1u << lane);
  const int K = x.K;
  const bool valid = c < INFINITY;
  const int nvalid = __popc(vm);
  if (__any_sync(FULL, valid && !(isfinite(F) && isfinite(g)))) {
    st.tfl |= TRACE_NONFINITE | TRACE_SEARCH_UNCONVERGED;
    st.bits |= SS_FINISHED;
    return;
  }
  // ---- sign changes against the immediate left neighbour ----
  double cl = __shfl_up_sync(FULL, c, 1), Fl = __shfl_up_sync(FULL, F, 1);
  bool exl = __shfl_up_sync(FULL, exact, 1);
  const bool vl = lane >= 1 ? lane - 1 < nvalid : (st.bits & SS_HAVE1) != 0;
  if (lane == 0) {
    cl = st.c1;
    Fl = st.F1;
    exl = (st.bits & SS_EX1) != 0;
  }
  const bool sc = valid && vl && (signbit(Fl) != signbit(F));  // +0 counts as positive
  const unsigned scm = __ballot_sync(FULL, sc);
  const int myseg = st.nseg + __popc(scm & le);
  Sample me{c, static_cast<float>(g), static_cast<float>(M),
            myseg | (exact ? (1 << 29) : 0) | (signbit(F) ? (1 << 30) : 0)};
  // ---- regular samples and their two regular predecessors ----
  const bool reg = valid && !(vl && c - cl < 1e-6 * c);
  const unsigned rmask = __ballot_sync(FULL, reg);
  const unsigned m1 = rmask & lt;
  const int j1 = m1 ? 31 - __clz(m1) : -1;
  const unsigned m2 = j1 >= 0 ? (m1 & ~(1u << j1)) : 0u;
  const int j2 = m2 ? 31 - __clz(m2) : -1;
  Sample P1 = shfl_sample(me, j1 & 31), P2 = shfl_sample(me, j2 & 31);
  bool hp1 = j1 >= 0, hp2 = j2 >= 0;
  if (j1 < 0) {
    P1 = st.R1; hp1 = (st.bits & SS_HR1) != 0;
    P2 = st.R2; hp2 = (st.bits & SS_HR2) != 0;
  } else if (j2 < 0) {
    P2 = st.R1; hp2 = (st.bits & SS_HR1) != 0;
  }
  // ---- same-sign troughs: V-shaped shape-feature minima, log-magnitude dips ----
  bool tr = false, trm_ = false;
  if (reg && hp1 && hp2 && sample_segment(P2) == myseg && sample_segment(P1) == myseg) {
    const double sgn = sample_sign(P1);
    tr = trough_may_hide_roots(P2.c, P1.c, c, sgn * P2.g, sgn * P1.g, sgn * static_cast<float>(g),
                               pair_noise(single, P2, P1), pair_noise(single, P1, me));
    if (!tr) trm_ = magnitude_dip(P2.c, P1.c, c, P2.M, P1.M, static_cast<float>(M)) > MDIP;
    tr = tr || trm_;
  }
  const unsigned trm = __ballot_sync(FULL, tr), mmode = __ballot_sync(FULL, trm_);
  unsigned events = scm | trm;
  while (events && st.nbr < K) {
    const int i = __ffs(events) - 1;
    events &= events - 1;
    if ((scm >> i) & 1u) {
      if (lane == i) put_bracket(x.slot, st.nbr, cl, c, exl ? Fl : NAN, exact ? F : NAN);
      ++st.nbr;
    } else {
      double x0 = __shfl_sync(FULL, P2.c, i), x1 = __shfl_sync(FULL, P1.c, i);
      const double x2 = __shfl_sync(FULL, c, i);
      const double sgn = (__shfl_sync(FULL, P1.seg, i) >> 30) & 1 ? -1. : 1.;
      double sa = sgn * __shfl_sync(FULL, P2.g, i), ma = __shfl_sync(FULL, P2.M, i);
      const double sb = sgn * __shfl_sync(FULL, g, i), mb = __shfl_sync(FULL, M, i);
      if (x0 < st.zoom_right) {  // overlaps the previous window: start at its middle sample
        x0 = x1;
        sa = sgn * __shfl_sync(FULL, P1.g, i);
        ma = __shfl_sync(FULL, P1.M, i);
      }
      st.zoom_right = x2;
      const int mode = (mmode >> i) & 1u;
      bool dismissed = false;
      if constexpr (single) {
        unsigned long long se = 0;
        dismissed = screen_trough32<WAVE>(view, static_cast<float>(x.w), x0, x2, sa, sb, ma, mb, sgn, mode, lane,
                                          se);
        ctr.evals += se;
        ctr.evals32 += se;
        ctr.steps += se * x.nsteps;
        ctr.steps32 += se * x.nsteps;
      }
      if (!dismissed) {
        unsigned long long ze = 0;
        st.nbr = zoom_trough<WAVE>(view64, x.w, x0, x2, sa, sb, ma, mb, sgn, mode, d.tol, x.slot, st.nbr, K, lane,
                                   ze);
        ctr.evals += ze;
        ctr.steps += ze * x.nsteps;
        ++ctr.zooms;
      }
    }
  }
  // ---- carries ----
  st.nseg += __popc(scm);
  const int last = nvalid - 1;
  st.c1 = __shfl_sync(FULL, c, last);
  st.F1 = __shfl_sync(FULL, F, last);
  st.bits = (st.bits & ~SS_EX1) | SS_HAVE1 | (__shfl_sync(FULL, exact, last) ? SS_EX1 : 0);
  if (rmask) {
    const int h1 = 31 - __clz(rmask);
    const unsigned rest = rmask & ~(1u << h1);
    const Sample n1 = shfl_sample(me, h1);
    const Sample n2 = shfl_sample(me, rest ? 31 - __clz(rest) : 0);
    if (rest) {
      st.R2 = n2;
      st.bits |= SS_HR2;
    } else {
      st.R2 = st.R1;
      st.bits = (st.bits & ~SS_HR2) | ((st.bits & SS_HR1) ? SS_HR2 : 0);
    }
    st.R1 = n1;
    st.bits |= SS_HR1;
  }
}

// The end of a trace's scan: the last-cell check and the brackets published
// for refinement.
template <class T, int WAVE>
__device__ __forceinline__ void scan_finish(const Dev &d, const TraceCtx &x, ScanState &st, const LayerView<T> &view,
                                            const LayerView<double> &view64, int lane, ScanCounters &ctr) {
  if ((st.bits & SS_FINISHED) && st.nbr < x.K && !(st.tfl & TRACE_SEARCH_UNCONVERGED) && (st.bits & SS_HR1) &&
      (st.bits & SS_HR2) && st.R2.c < st.R1.c && st.zoom_right <= st.R2.c &&
      sample_segment(st.R1) == sample_segment(st.R2))
    st.nbr = last_cell<T, WAVE>(view, view64, x.w, st.R2, st.R1, d.tol, x.slot, st.nbr, x.K, lane, x.nsteps,
                                ctr.evals, ctr.evals32, ctr.steps, ctr.steps32, ctr.zooms);
  if (lane == 0) {
    d.nbr[x.t] = st.nbr;
    if (st.tfl) atomicOr(&d.tflags[x.t], st.tfl);
  }
  if (!(st.tfl & TRACE_SEARCH_UNCONVERGED)) {
    int base = 0;
    if (lane == 0) base = atomicAdd(&d.ctr[C_NREFINE], st.nbr);
    base = __shfl_sync(FULL, base, 0);
    for (int i = lane; i < st.nbr; i += 32) d.refine_list[base + i] = x.t * d.KB + i;
  }
  __syncwarp();
}

__device__ __forceinline__ void scan_counters_flush(const Dev &d, const ScanCounters &ctr, int lane) {
  if (lane == 0 && d.stats) {
    if (ctr.evals) atomicAdd(&d.stats[0], ctr.evals);
    if (ctr.steps) atomicAdd(&d.stats[2], ctr.steps);
    if (ctr.evals32) atomicAdd(&d.stats[1], ctr.evals32);
    if (ctr.steps32) atomicAdd(&d.stats[3], ctr.steps32);
    if (ctr.zooms) atomicAdd(&d.stats[5], ctr.zooms);
  }
}

// ---------------------------------------------------------------------------
// scan<T, WAVE>: the fused persistent kernel, one warp per trace.
// Shared memory per warp: EVAL_ROWS * Ls values of T (model table) + 32 doubles
// (merge buffer).
// ---------------------------------------------------------------------------
template <class T, int WAVE>
__global__ void __launch_bounds__(128, (sizeof(T) == 4 && WAVE == 1) ? MD200_SCAN_MIN_BLOCKS_LOVE32
                                                                      : MD200_SCAN_MIN_BLOCKS)
    scan(Dev d, const int *list, int cursor_id, int count_id,
                                                                   int resume = 0) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const size_t tab_bytes = (static_cast<size_t>(EVAL_ROWS) * d.Ls * sizeof(T) + 15) & ~size_t(15);
  unsigned char *mine = smem_raw + static_cast<size_t>(wib) * (tab_bytes + 32 * sizeof(double));
  T *tab = reinterpret_cast<T *>(mine);
  double *mbuf = reinterpret_cast<double *>(mine + tab_bytes);
  ScanCounters ctr;
  const double step = 1. / d.density;
  constexpr bool single = sizeof(T) == 4;

  for (;;) {
    int q = 0;
    if (lane == 0) q = atomicAdd(&d.ctr[cursor_id], 1);
    q = __shfl_sync(FULL, q, 0);
    if (q >= *(volatile int *)&d.ctr[count_id]) break;
    const TraceCtx x = trace_ctx(d, list[q]);
    // stage the model's recurrence rows (16-byte cp.async, coalesced)
    {
      const T *src = layer_table<T>(d, x.b);
      const int n16 = static_cast<int>((static_cast<size_t>(EVAL_ROWS) * d.Ls * sizeof(T)) / 16);
      for (int i = lane; i < n16; i += 32)
        cp_async16(reinterpret_cast<unsigned char *>(tab) + 16 * i,
                   reinterpret_cast<const unsigned char *>(src) + 16 * i);
      cp_async_wait_all();
      __syncwarp();
    }
    const LayerView<T> view = make_view<T>(tab, d.Ls, d.mL[x.b], d.mwater[x.b]);
    // FP64 view for zooms and FP64 samples of the single-precision scan (global
    // memory, L1/L2-resident); the FP64 scan reads its shared-memory copy
    LayerView<double> view64;
    if constexpr (single) view64 = global_view(d, x.b);
    else view64 = *reinterpret_cast<const LayerView<double> *>(&view);
    // a fresh trace, or (resume) one the split scan handed over mid-way
    ScanState st = resume ? d.sp_state[x.t] : scan_start(d, x);
    int kfrom = 0;  // this lane's knot interval (scan_point)
    while (st.nbr < x.K && !(st.bits & SS_FINISHED)) {
      double c;
      const unsigned vm = scan_positions(x, st, step, lane, mbuf, kfrom, c);
      if (!vm) {
        st.bits |= SS_FINISHED;  // the window is exhausted
        break;
      }
      const bool valid = c < INFINITY;
      const int nv = __popc(vm);
      double F, g, M;
      bool exact;
      if constexpr (single) {
        bool near_cut;
        const float c32 = scan_position32(c, x.hi, near_cut);
        float F32, g32, M32;
        scan_eval<float, WAVE, 1>(view, static_cast<float>(x.w), &c32, &F32, &g32, &M32);
        F = F32;
        g = g32;
        M = M32;
        ctr.evals += nv;
        ctr.evals32 += nv;
        ctr.steps += static_cast<unsigned long long>(nv) * x.nsteps;
        ctr.steps32 += static_cast<unsigned long long>(nv) * x.nsteps;
        const bool redo = scan_complete32<WAVE>(view64, x.w, x.tail, c, valid, near_cut, F, g, M, exact);
        const int nr = __popc(__ballot_sync(FULL, redo));
        ctr.evals += nr;
        ctr.steps += static_cast<unsigned long long>(nr) * x.nsteps;
      } else {
        double c64 = valid ? c : 1.;
        scan_eval<double, WAVE, 1>(view, x.w, &c64, &F, &g, &M);
        exact = true;
        ctr.evals += nv;
        ctr.steps += static_cast<unsigned long long>(nv) * x.nsteps;
      }
      scan_bookkeep<T, WAVE>(d, x, st, view, view64, lane, c, F, g, M, exact, vm, ctr);
    }
    scan_finish<T, WAVE>(d, x, st, view, view64, lane, ctr);
  }
  scan_counters_flush(d, ctr, lane);
}

// One refinement sample.  F is the secular value as the recurrence returns it,
// renormalised by a power of two at every layer; (g, l) stands for g 2^l, with
// g the shape feature F / |e| and l the base-2 log-magnitude of the
// unnormalised vector less the evanescent factor exp(sum r h) -- together the
// function on one smooth scale.  Near a root where the whole vector vanishes (a
// mode trapped under an evanescent layer) the renormalisation rescales F by its
// own magnitude: F turns step-like (about +-0.4 on either side of the root),
// interpolation on it fails and the bracket closes by bisection to a midpoint.
// Ratios of two samples are therefore taken on the g 2^l scale; bracket ends
// carried over from the scan have no l (NaN), and ratios involving them use F.
struct RootSample {
  double F, g, l;
};
__device__ __forceinline__ double sample_ratio(const RootSample &x, const RootSample &y) {
  const double dl = x.l - y.l;
  return isnan(dl) ? x.F / y.F : (x.g / y.g) * exp2(dl);
}
__device__ __forceinline__ RootSample root_sample(const LayerView<double> &m, int wave, double w, double c) {
  RootSample r;
  double lev;
  r.F = secular<double, double>(m, wave, w / c, w, &r.g, &r.l, &lev);
  r.l -= lev;
  return r;
}

// Refinement of one bracket [a, b] to the reference's stopping width
// max(16 eps |x|, min(w/64, tol |x| / 8)) by Brent-Dekker
// (cpp/common/refinement.hpp:341-396) on RootSamples, written as a state
// machine: brent_advance either asks for the function at a point or finishes,
// brent_absorb takes the sample.  End values unknown in FP64 (NaN: brackets of
// the FP32 scan) are asked for first.  At most BRENT_MAX_EVALS evaluations.
constexpr int BRENT_MAX_EVALS = 162;
enum BrentStep { BRENT_EVAL = 0, BRENT_DONE = 1, BRENT_NO_BRACKET = 2 };
struct BrentState {
  double a, b, c, dd, e, stop;
  RootSample sa, sb, sc;
  int pending;  // bit 0: f(a) unknown, bit 1: f(b) unknown
  int evals;
  bool confirm, started, failed;
};

__device__ __forceinline__ void brent_init(BrentState &st, double a, double b, double fa, double fb) {
  st.a = a;
  st.b = b;
  st.c = b;
  st.dd = st.e = st.stop = 0.;
  st.sa = RootSample{fa, fa, NAN};
  st.sb = RootSample{fb, fb, NAN};
  st.sc = RootSample{0., 0., NAN};
  st.pending = (isfinite(fa) ? 0 : 1) | (isfinite(fb) ? 0 : 2);
  st.confirm = st.pending != 0;
  st.started = st.failed = false;
  st.evals = 0;
}

__device__ __forceinline__ void brent_absorb(BrentState &st, const RootSample &smp) {
  ++st.evals;
  if (st.pending & 1) {
    st.sa = smp;
    st.pending &= ~1;
  } else if (st.pending & 2) {
    st.sb = smp;
    st.pending &= ~2;
  } else {
    st.sb = smp;
    if (!isfinite(smp.F)) st.failed = true;
  }
}

// BRENT_EVAL: evaluate at *x next.  BRENT_DONE: *root (NaN when refinement
// failed).  BRENT_NO_BRACKET: the confirmed FP64 ends have one sign.
__device__ __forceinline__ int brent_advance(BrentState &st, double tol, double *x, double *root) {
  if (st.pending) {
    *x = (st.pending & 1) ? st.a : st.b;
    return BRENT_EVAL;
  }
  *root = NAN;
  if (st.failed) return BRENT_DONE;
  double a = st.a, b = st.b, c = st.c, dd = st.dd, e = st.e;
  RootSample sa = st.sa, sb = st.sb, sc = st.sc;
  if (!st.started) {
    st.started = true;
    if (st.confirm && signbit(sa.F) == signbit(sb.F)) return BRENT_NO_BRACKET;
    if (a == b) {
      if (sa.F == 0.) *root = a;
      return BRENT_DONE;
    }
    if (!isfinite(sa.F) || !isfinite(sb.F) || ((sa.F < 0.) == (sb.F < 0.) && sa.F != 0. && sb.F != 0.))
      return BRENT_DONE;
    if (sa.F == 0.) { *root = a; return BRENT_DONE; }
    if (sb.F == 0.) { *root = b; return BRENT_DONE; }
    const double big = fmax(fabs(a), fabs(b));
    st.stop = fmax(16. * 2.220446049250313e-16 * big, fmin((b - a) / 64., .125 * tol * big));
    c = b;
    sc = sb;
    dd = e = b - a;
  }
  if (st.evals >= BRENT_MAX_EVALS) return BRENT_DONE;
  if ((sb.F < 0.) == (sc.F < 0.)) {
    c = a;
    sc = sa;
    e = dd = b - a;
  }
  if (fabs(sample_ratio(sc, sb)) < 1.) {  // |f(c)| < |f(b)|
    a = b; sa = sb;
    b = c; sb = sc;
    c = a; sc = sa;
  }
  if (sb.F == 0.) { *root = b; return BRENT_DONE; }
  const double mid = .5 * (c - b), half = .5 * st.stop;
  if (fabs(c - b) <= st.stop) {
    // converged bracket [b, c], f(b) and f(c) of opposite signs: its secant
    // point is second order in the width and needs no evaluation (group
    // velocities of some roots move by 1e-7 per 1e-11 of root error, so the
    // midpoint's error of up to stop / 2 would show in them)
    const double s = b - (c - b) / (sample_ratio(sc, sb) - 1.);
    *root = (isfinite(s) && (s - b) * (s - c) <= 0.) ? s : .5 * (b + c);
    return BRENT_DONE;
  }
  if (fabs(e) >= half && fabs(sample_ratio(sa, sb)) > 1.) {
    const double s = sample_ratio(sb, sa);
    double p, q;
    if (a == c) {
      p = 2. * mid * s;
      q = 1. - s;
    } else {
      const double qa = sample_ratio(sa, sc), r = sample_ratio(sb, sc);
      p = s * (2. * mid * qa * (qa - r) - (b - a) * (r - 1.));
      q = (qa - 1.) * (r - 1.) * (s - 1.);
    }
    if (p > 0.) q = -q; else p = -p;
    const double old = e;
    e = dd;
    const double ratio = p / q;
    if (isfinite(ratio) && 2. * p < fmin(3. * mid * q - fabs(half * q), fabs(old * q))) dd = ratio;
    else { dd = mid; e = mid; }
  } else {
    dd = mid;
    e = mid;
  }
  a = b;
  sa = sb;
  b += fabs(dd) > half ? dd : (mid > 0. ? half : -half);
  st.a = a; st.b = b; st.c = c; st.dd = dd; st.e = e;
  st.sa = sa; st.sb = sb; st.sc = sc;
  *x = b;
  return BRENT_EVAL;
}

// ---------------------------------------------------------------------------
// refine: one bracket per lane, lanes refilled from the bracket list.
// Brackets converge in different numbers of evaluations; with one fixed bracket
// per thread half the lanes of a warp idled on average.  Here every loop
// iteration is one secular evaluation for all lanes that have work (one call
// site), and a lane whose bracket finishes takes the next one from the list
// (warp-aggregated atomic on C_REFINE_CURSOR) in the same iteration.  Each
// bracket follows the same arithmetic as on its own, so results do not depend
// on the schedule.
// ---------------------------------------------------------------------------
struct RefineLane {
  BrentState st;
  LayerView<double> m;
  double w;
  double *sl;
  int id, t;
  bool eval, exhausted;
};

__device__ __forceinline__ void refine_step(Dev &d, RefineLane &L, double *x, unsigned long long &count) {
  if (L.id < 0 || L.eval) return;
  double root;
  const int r = brent_advance(L.st, d.tol, x, &root);
  if (r == BRENT_EVAL) {
    L.eval = true;
    return;
  }
  L.sl[4] = r == BRENT_DONE ? root : NAN;
  if (r == BRENT_NO_BRACKET) {  // the FP32 scan's sign change does not hold in FP64
    atomicOr(&d.tflags[L.t], INTERNAL_REPAIR);
  } else {
    if (!isfinite(root)) atomicOr(&d.tflags[L.t], TRACE_REFINEMENT_FAILED);
    ++count;
  }
  L.id = -1;
}

__device__ __forceinline__ void refine_fetch(Dev &d, RefineLane &L, int end, int lane) {
  const bool need = L.id < 0 && !L.exhausted;
  const unsigned nm = __ballot_sync(FULL, need);
  if (!nm) return;
  const int leader = __ffs(nm) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(&d.ctr[C_REFINE_CURSOR], __popc(nm));
  base = __shfl_sync(FULL, base, leader);
  if (!need) return;
  const int i = base + __popc(nm & lanemask_lt());
  if (i >= end) {
    L.exhausted = true;
    return;
  }
  L.id = d.refine_list[i];
  L.t = L.id / d.KB;
  L.m = global_view(d, d.tr_model[L.t]);
  L.w = TWO_PI / d.tr_period[L.t];
  L.sl = d.slot + static_cast<size_t>(L.id) * SLOT;
  brent_init(L.st, L.sl[0], L.sl[1], L.sl[2], L.sl[3]);
}

#ifndef MD200_REFINE_MIN_BLOCKS
#define MD200_REFINE_MIN_BLOCKS 4
#endif
__global__ void __launch_bounds__(128, MD200_REFINE_MIN_BLOCKS) refine(Dev d) {
  const int lane = threadIdx.x & 31;
  const int end = d.ctr[C_NREFINE];
  unsigned long long evals = 0, steps = 0, count = 0;
  RefineLane L;
  L.id = -1;
  L.exhausted = false;
  for (;;) {
    double x = 0.;
    L.eval = false;
    refine_step(d, L, &x, count);
    refine_fetch(d, L, end, lane);
    refine_step(d, L, &x, count);
    refine_fetch(d, L, end, lane);
    refine_step(d, L, &x, count);
    if (__all_sync(FULL, !L.eval && L.exhausted)) break;
    if (L.eval) {
      const RootSample smp = root_sample(L.m, d.wave, L.w, x);  // the one evaluation site
      brent_absorb(L.st, smp);
      ++evals;
      steps += layer_steps(L.m.L, L.m.water);
    }
  }
  if (d.stats && (evals || count)) {
    atomicAdd(&d.stats[0], evals);
    atomicAdd(&d.stats[2], steps);
    atomicAdd(&d.stats[4], count);
  }
}

// Every pass after the first re-solves a set of traces: its scan appends
// brackets to the refine list and its assembly roots to the group list.  The
// previous pass's entries are consumed by then, so each pass restarts both lists
// at zero and needs at most one pass's capacity (KB brackets and nmodes roots per
// trace).  Called by the first thread of the pass's collecting kernel.
__device__ __forceinline__ void restart_refine_list(const Dev &d) {
  d.ctr[C_NREFINE] = d.ctr[C_REFINE_BEGIN] = d.ctr[C_REFINE_CURSOR] = 0;
}
__device__ __forceinline__ void restart_lists(const Dev &d) {
  restart_refine_list(d);
  d.ctr[C_NGROUP] = d.ctr[C_GROUP_BEGIN] = 0;
}

// ---------------------------------------------------------------------------
// collect_repairs: traces whose FP32 scan FP64 did not confirm.
// ---------------------------------------------------------------------------
__global__ void collect_repairs(Dev d) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t == 0) restart_refine_list(d);
  if (t >= d.n_traces) return;
  const unsigned fl = d.tflags[t];
  if (fl & INTERNAL_REPAIR) {
    const int pos = atomicAdd(&d.ctr[C_NREPAIR], 1);
    d.repair_list[pos] = t;
    d.tflags[t] = (fl & ~(INTERNAL_REPAIR | TRACE_REFINEMENT_FAILED)) | TRACE_FP64_REPAIR;
    d.nbr[t] = 0;
    if (d.stats) atomicAdd(&d.stats[7], 1ULL);
  }
}

// ---------------------------------------------------------------------------
// collect_fallback: traces the first search could not finish -- a non-finite
// value (the FP32 range, say), or the scan-point limit reached before the trace
// held all its brackets -- re-scanned in FP64 with the larger limit
// JMAX_FALLBACK (the reference escalates such traces to its adaptive ladder and
// dense grid, cpp/cpu/solver.cpp:254-370,517-584).  Their earlier roots are
// taken out of the counters; assemble() reports them at LEVEL_FALLBACK with
// TRACE_ADAPTIVE_FALLBACK.
// ---------------------------------------------------------------------------
__global__ void collect_fallback(Dev d) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t == 0) restart_lists(d);
  if (t >= d.n_traces) return;
  const int b = d.tr_model[t];
  if (d.mstate[b] != 0) return;
  const unsigned fl = d.tflags[t];
  const bool capped = (fl & TRACE_WORKSPACE_LIMIT) && d.nbr[t] < d.tr_modes[t] + 2;
  if (!(fl & TRACE_SEARCH_UNCONVERGED) && !capped) return;
  const int pos = atomicAdd(&d.ctr[C_NREPAIR], 1);
  d.repair_list[pos] = t;
  // (an FP64 re-solve: in an FP32-scan engine also an FP64 repair, which the
  // continuity recheck does not re-scan)
  d.tflags[t] = TRACE_ADAPTIVE_FALLBACK | (d.fp32 ? TRACE_FP64_REPAIR : 0u);
  d.nbr[t] = 0;
  if (d.stats) {
    const int nm = d.tr_modes[t], s = d.tr_stride[t];
    const size_t o = static_cast<size_t>(d.tr_out[t]);
    int finite = 0;
    for (int k = 0; k < nm; ++k) finite += isfinite(d.vel[o + static_cast<size_t>(k) * s]);
    if (finite) atomicAdd(&d.stats[10], static_cast<unsigned long long>(-finite));
    if (fl & TRACE_SEARCH_UNCONVERGED) atomicAdd(&d.stats[8], static_cast<unsigned long long>(-1LL));
    atomicAdd(&d.stats[16], 1ULL);
  }
}

// ---------------------------------------------------------------------------
// assemble: one thread per trace.
// ---------------------------------------------------------------------------
// With `list`, only the traces list[0 .. ctr[count_id]) (re-solved traces)
// are assembled again; their previous roots are taken out of the root count.
__global__ void assemble(Dev d, const int *list = nullptr, int count_id = 0) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (list) {
    if (t >= *(volatile int *)&d.ctr[count_id]) return;
    t = list[t];
  } else if (t >= d.n_traces) {
    return;
  }
  const int b = d.tr_model[t];
  const int nm = d.tr_modes[t], T = d.tr_stride[t];  // modes of this trace, stride between them
  const size_t out0 = static_cast<size_t>(d.tr_out[t]);
  const int state = d.mstate[b];
  if (state != 0) {
    for (int m = 0; m < nm; ++m) d.vel[out0 + static_cast<size_t>(m) * T] = NAN;
    d.oflags[t] = 0;
    d.olevels[t] = state;
    d.ocounts[t] = 0;
    if (d.group)
      for (int m = 0; m < nm; ++m) {
        d.grp[out0 + static_cast<size_t>(m) * T] = NAN;
        d.gflags[out0 + static_cast<size_t>(m) * T] = GROUP_MISSING_ROOT;
      }
    return;
  }
  unsigned fl = d.tflags[t];
  const int nbr = d.nbr[t];
  // The refined roots sit in the root field of the trace's bracket slots (at most
  // K = nmodes + 2 of them: the scan stops at K brackets).  They are ordered in
  // place there, so every mode count the engine accepts (up to 256 + 2 guards)
  // keeps all of its roots; nothing reads a slot's bracket after assembly (a
  // re-solved trace is scanned into its slots afresh).
  double *rs = d.slot + static_cast<size_t>(t) * d.KB * SLOT + 4;
  auto r = [rs](int i) -> double & { return rs[static_cast<size_t>(i) * SLOT]; };
  bool failed = (fl & (TRACE_SEARCH_UNCONVERGED | INTERNAL_REPAIR)) != 0;
  for (int s = 0; s < nbr && !failed; ++s)
    if (!isfinite(r(s))) failed = true;
  int n = 0;
  if (!failed) {
    // insertion sort (brackets arrive in velocity order: nearly sorted already)
    for (int i = 1; i < nbr; ++i) {
      const double x = r(i);
      int j = i;
      while (j > 0 && r(j - 1) > x) {
        r(j) = r(j - 1);
        --j;
      }
      r(j) = x;
    }
    // exact duplicates (an exact zero shared by two brackets) collapse to one root
    for (int i = 0; i < nbr; ++i)
      if (n == 0 || r(i) != r(n - 1)) r(n++) = r(i);
  }
  const double lo = d.mlo[b], hi = d.mhi[b];
  const LayerView<double> m = global_view(d, b);
  const double vs_hs = layer_table<double>(d, b)[8 * d.Ls + m.L - 1];
  const double w = TWO_PI / d.tr_period[t];
  int level = d.fp32 ? ((fl & TRACE_FP64_REPAIR) ? LEVEL_REPAIRED : LEVEL_FP32) : LEVEL_FP64;
  if (fl & TRACE_ADAPTIVE_FALLBACK) level = LEVEL_FALLBACK;
  if (fl & TRACE_CONTINUATION_APPROXIMATE) level = LEVEL_CONTINUATION;
  int count = n;
  if (failed) {
    fl |= TRACE_SEARCH_UNCONVERGED;
    count = -1;
    level = -1;
    n = 0;
  }
  for (int i = 1; i < n; ++i)
    if (r(i) - r(i - 1) <= d.close_rtol * r(i)) fl |= TRACE_CLOSE_ROOT_RISK;
  for (int mo = 0; mo < nm; ++mo) {
    double root = mo < n ? r(mo) : NAN;
    if (isfinite(root) && root >= .99 * vs_hs) fl |= TRACE_NEAR_CUTOFF;
    if (isfinite(root) && d.accept < 1.) {
      const double v = eval64(m, d.wave, w, root, nullptr);
      if (!isfinite(v) || fabs(v) > d.accept) {
        root = NAN;
        fl |= TRACE_F_REJECTED;
      }
    }
    const size_t cell = out0 + static_cast<size_t>(mo) * T;
    d.vel[cell] = root;
    if (d.group) {
      if (!isfinite(root)) {
        d.grp[cell] = NAN;
        d.gflags[cell] = GROUP_MISSING_ROOT;
      } else {
        // neighbour-midpoint window and close-root test (cpp/cpu/solver.cpp:96-103)
        const double c = r(mo);
        const double wl = mo ? .5 * (r(mo - 1) + c) : lo;
        const double wh = mo + 1 < n ? .5 * (c + r(mo + 1)) : hi;
        const bool close = (mo && c - r(mo - 1) <= d.close_rtol * c) ||
                           (mo + 1 < n && r(mo + 1) - c <= d.close_rtol * r(mo + 1));
        d.gwin[2 * cell] = wl;
        d.gwin[2 * cell + 1] = wh;
        if (close) {
          d.grp[cell] = NAN;
          d.gflags[cell] = GROUP_CLOSE_ROOT;
        } else {
          d.gflags[cell] = 0;
          const int pos = atomicAdd(&d.ctr[C_NGROUP], 1);
          d.group_list[pos] = t * d.KB + mo;
        }
      }
    }
  }
  d.oflags[t] = fl & ~INTERNAL_MASK;
  d.olevels[t] = level;
  d.ocounts[t] = count;
  if (d.stats) {
    if (!list) atomicAdd(&d.stats[11], 1ULL);
    if (failed) atomicAdd(&d.stats[8], 1ULL);
    int finite = 0;
    for (int mo = 0; mo < nm && mo < n; ++mo) finite += isfinite(d.vel[out0 + static_cast<size_t>(mo) * T]);
    if (finite) atomicAdd(&d.stats[10], static_cast<unsigned long long>(finite));
  }
}

// ---------------------------------------------------------------------------
// continuity_screen: one thread per trace of an FP32-scan run, after assembly.
// The rules of the reference's screen (cpp/cpu/continuity_screen.hpp:8-67) on
// the phase velocities as float32 values (the precision of the reference's
// FP32 results, which its screen sees as float32):
//   ENVELOPE (16)   with the neighbouring periods of the model (in period order)
//                   within a log step of 0.25, a mode with roots at both that is
//                   missing here or outside [0.95 min, 1.05 max] of them;
//   CLOSE_FP32 (32) adjacent modes within 16 float32 ULPs;
//   PREDICTION (64) a continuation prediction marked for review;
//   NO_BILATERAL (8) until some mode has roots at both neighbours.
// Suspects (16 | 32 | 64) are REVIEWED (1) and queued for an FP64 re-scan (the
// repair list) unless FP64 already re-solved them in this run; their roots and
// count are kept in d.cold / d.ccount for continuity_finish, their old roots are
// taken out of the root count and their group-velocity entries re-queued.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double log_step(double target, double anchor) {
  // cpp/common/continuation.hpp:12-15
  return fabs(target - anchor) < .5 * anchor ? log1p((target - anchor) / anchor) : log(target) - log(anchor);
}
__device__ __forceinline__ double as_float(double x) { return static_cast<double>(static_cast<float>(x)); }

// The screen's flags of one trace: its nm roots at vel[o + k s], those of its
// neighbouring periods at vel[ol + k sl] and vel[orr + k sr] (read only when
// `interior`), its prediction word.  `single`: the roots are compared as
// float32 values and the CLOSE_FP32 rule applies (the reference's screen of
// float32 results); `bilateral`: the envelope rule is on.
__device__ __forceinline__ unsigned screen_flag(const double *vel, size_t o, int s, size_t ol, int sl, size_t orr,
                                                int sr, bool interior, int nm, unsigned pred, bool single,
                                                bool bilateral) {
  unsigned flag = bilateral ? CONT_NO_BILATERAL : 0u;
  interior = interior && bilateral;
  if (interior || (bilateral && single && nm > 1)) {
    double prev = NAN;
    for (int k = 0; k < nm; ++k) {
      double c = vel[o + static_cast<size_t>(k) * s];
      if (single) c = as_float(c);
      if (interior) {
        double cl = vel[ol + static_cast<size_t>(k) * sl], cr = vel[orr + static_cast<size_t>(k) * sr];
        if (single) cl = as_float(cl), cr = as_float(cr);
        if (isfinite(cl) && isfinite(cr)) {
          flag &= ~CONT_NO_BILATERAL;
          if (!isfinite(c) || c < .95 * fmin(cl, cr) || c > 1.05 * fmax(cl, cr)) flag |= CONT_ENVELOPE;
        }
      }
      if (single && k && isfinite(c) && isfinite(prev)) {
        const unsigned x = __float_as_uint(static_cast<float>(c)), y = __float_as_uint(static_cast<float>(prev));
        if ((x > y ? x - y : y - x) <= 16u) flag |= CONT_CLOSE_FP32;
      }
      prev = c;
    }
  }
  if (pred & PRED_REVIEW) flag |= CONT_PREDICTION;
  return flag;
}

// The screen alone on a [B][K][T] result (the reference's module function,
// cpp/cpu/continuity_screen.hpp:8-67): one thread per (model, period rank);
// `order` is the period order the host chose (identity for ascending periods).
__global__ void continuity_screen_plain(const double *periods, const int *order, int T, const double *vel, int B,
                                        int K, const unsigned *pred, int single, int bilateral,
                                        unsigned char *out, int *suspect) {
  const long long q = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (q >= static_cast<long long>(B) * T) return;
  const int b = static_cast<int>(q / T), j = static_cast<int>(q - static_cast<long long>(b) * T);
  const int f = order[j], l = order[j > 0 ? j - 1 : j], r = order[j + 1 < T ? j + 1 : j];
  const bool interior = j > 0 && j + 1 < T && log_step(periods[r], periods[l]) <= .25;
  const size_t base = static_cast<size_t>(b) * K * T;
  const unsigned flag = screen_flag(vel, base + f, T, base + l, T, base + r, T, interior, K,
                                    pred ? pred[static_cast<size_t>(b) * T + f] : 0u, single != 0, bilateral != 0);
  out[static_cast<size_t>(b) * T + f] = static_cast<unsigned char>(flag);
  if (flag & (CONT_ENVELOPE | CONT_CLOSE_FP32 | CONT_PREDICTION)) *suspect = 1;
}

__global__ void continuity_screen(Dev d) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t == 0) restart_lists(d);
  if (t >= d.n_traces) return;
  const int b = d.tr_model[t];
  // the model's traces
  int first, count;
  if (d.ragged) {
    first = d.r_offsets[b];
    count = d.r_offsets[b + 1] - first;
  } else {
    first = b * d.T;
    count = d.T;
  }
  // neighbours in period order: the nearest shorter and longer periods
  const double p = d.tr_period[t];
  int l = -1, r = -1;
  double pl = -INFINITY, pr = INFINITY;
  for (int j = 0; j < count; ++j) {
    const double q = d.tr_period[first + j];
    if (q < p && q > pl) { pl = q; l = first + j; }
    if (q > p && q < pr) { pr = q; r = first + j; }
  }
  const bool interior = l >= 0 && r >= 0 && log_step(pr, pl) <= .25;
  const int nm = d.tr_modes[t];
  const size_t o = static_cast<size_t>(d.tr_out[t]);
  const int s = d.tr_stride[t];
  unsigned flag = screen_flag(d.vel, o, s, interior ? static_cast<size_t>(d.tr_out[l]) : 0, interior ? d.tr_stride[l] : 0,
                              interior ? static_cast<size_t>(d.tr_out[r]) : 0, interior ? d.tr_stride[r] : 0, interior,
                              nm, d.pred ? d.pred[t] : 0u, true, true);
  const bool suspect = (flag & (CONT_ENVELOPE | CONT_CLOSE_FP32 | CONT_PREDICTION)) != 0;
  if (suspect) flag |= CONT_REVIEWED;
  if (d.cflags) d.cflags[t] = static_cast<unsigned char>(flag);
  const unsigned fl = d.tflags[t];
  if (!suspect || d.mstate[b] != 0 || (fl & TRACE_FP64_REPAIR)) return;  // FP64 already solved it
  if (d.cold) {  // (by trace: tr_modes[t] <= nmodes)
    double *keep = d.cold + static_cast<size_t>(t) * d.nmodes;
    for (int k = 0; k < nm; ++k) keep[k] = d.vel[o + static_cast<size_t>(k) * s];
    d.ccount[t] = d.ocounts[t];
  }
  const int pos = atomicAdd(&d.ctr[C_NREPAIR], 1);
  d.repair_list[pos] = t;
  d.tflags[t] = TRACE_FP64_REPAIR;  // the FP64 scan sets its own search flags afresh
  d.nbr[t] = 0;
  atomicAdd(&d.ctr[C_NSUSPECT], 1);
  if (d.stats) {
    int finite = 0;
    for (int k = 0; k < nm; ++k) finite += isfinite(d.vel[o + static_cast<size_t>(k) * s]);
    if (finite) atomicAdd(&d.stats[10], static_cast<unsigned long long>(-finite));
    if (fl & TRACE_SEARCH_UNCONVERGED) atomicAdd(&d.stats[8], static_cast<unsigned long long>(-1LL));
    atomicAdd(&d.stats[15], 1ULL);
  }
}

// continuity_finish: one thread per re-scanned suspect, after its FP64 re-solve.
// REPAIRED (2) when the root count or a root moved by more than the refinement
// tolerance (the reference adopts a review result under that test,
// python/modisp/_continuity.py:96-100); UNRESOLVED (4) when the FP64 search
// failed.
__global__ void continuity_finish(Dev d) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= *(volatile int *)&d.ctr[C_NREPAIR]) return;
  const int t = d.repair_list[i];
  const int nm = d.tr_modes[t];
  const size_t o = static_cast<size_t>(d.tr_out[t]);
  const int s = d.tr_stride[t];
  unsigned flag = d.cflags[t];
  if ((d.oflags[t] & TRACE_SEARCH_UNCONVERGED) || d.ocounts[t] < 0) {
    flag |= CONT_UNRESOLVED;
  } else {
    const double *kept = d.cold + static_cast<size_t>(t) * d.nmodes;
    bool changed = d.ocounts[t] != d.ccount[t];
    for (int k = 0; k < nm && !changed; ++k) {
      const double x = d.vel[o + static_cast<size_t>(k) * s], y = kept[k];
      if (isfinite(x) != isfinite(y)) changed = true;
      else if (isfinite(x) && fabs(x - y) > d.tol * fabs(x)) changed = true;
    }
    if (changed) flag |= CONT_REPAIRED;
  }
  d.cflags[t] = static_cast<unsigned char>(flag);
}

// ---------------------------------------------------------------------------
// group: one thread per root.  U = -F_k / F_omega from one forward-mode
// evaluation (value + two directional derivatives) at the refined root.
// ---------------------------------------------------------------------------
// 3 resident CTAs per SM (168 registers, a little spilling) measured 5-10 %
// faster than the uncapped 237-register build at 2 CTAs per SM
#ifndef MD200_GROUP_MIN_BLOCKS
#define MD200_GROUP_MIN_BLOCKS 3
#endif
__global__ void __launch_bounds__(128, MD200_GROUP_MIN_BLOCKS) group_velocity(Dev d) {
  const int n = d.ctr[C_NGROUP];
  unsigned long long steps = 0, count = 0;
  for (int i = d.ctr[C_GROUP_BEGIN] + blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int id = d.group_list[i];  // trace * KB + mode
    const int t = id / d.KB, mo = id - t * d.KB;
    const size_t cell = static_cast<size_t>(d.tr_out[t]) + static_cast<size_t>(mo) * d.tr_stride[t];
    const int b = d.tr_model[t];
    const LayerView<double> m = global_view(d, b);
    const double c = d.vel[cell];
    const double w = TWO_PI / d.tr_period[t];
    using D2 = Dual<double, 2>;
    D2 k, wd;
    k.v = w / c; k.d[0] = 1.; k.d[1] = 0.;
    wd.v = w; wd.d[0] = 0.; wd.d[1] = 1.;
    const D2 F = secular<D2, double>(m, d.wave, k, wd, nullptr);
    const double fk = F.d[0], fw = F.d[1];
    double u = -fk / fw;
    unsigned flag = 0;
    if (!isfinite(fk) || !isfinite(fw)) flag = GROUP_NONFINITE;
    else if (fw == 0. || !isfinite(u) || !(u > 0.)) flag = GROUP_ILL_CONDITIONED;
    d.grp[cell] = flag ? NAN : u;
    d.gflags[cell] = flag;
    steps += layer_steps(m.L, m.water);
    ++count;
  }
  if (d.stats && count) {
    atomicAdd(&d.stats[12], steps);
    atomicAdd(&d.stats[9], count);
  }
}

// ---------------------------------------------------------------------------
// group_roots: group velocities of one model's given ordered roots (the
// reference's review-group bridge, cpp/common/review_groups.hpp:9-34).  `tab` is
// a prepared [EVAL_ROWS][L] table.
// ---------------------------------------------------------------------------
__global__ void group_roots(const double *tab, int L, int water, int wave, double w,
                            const double *roots, int known, int modes, double close_rtol,
                            double *group, unsigned *flags) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= modes) return;
  if (j >= known) {
    group[j] = NAN;
    flags[j] = GROUP_MISSING_ROOT;
    return;
  }
  const double c = roots[j];
  if ((j && c - roots[j - 1] <= close_rtol * c) ||
      (j + 1 < known && roots[j + 1] - c <= close_rtol * roots[j + 1])) {
    group[j] = NAN;
    flags[j] = GROUP_CLOSE_ROOT;
    return;
  }
  // a packed root that is NaN or not positive is a missing root
  // (cpp/common/group_velocity.hpp:31): k = w / c would be meaningless
  if (!isfinite(c) || !(c > 0.)) {
    group[j] = NAN;
    flags[j] = GROUP_MISSING_ROOT;
    return;
  }
  const LayerView<double> m = make_view<double>(tab, L, L, water);
  using D2 = Dual<double, 2>;
  D2 k, wd;
  k.v = w / c; k.d[0] = 1.; k.d[1] = 0.;
  wd.v = w; wd.d[0] = 0.; wd.d[1] = 1.;
  const D2 F = secular<D2, double>(m, wave, k, wd, nullptr);
  const double u = -F.d[0] / F.d[1];
  unsigned flag = 0;
  if (!isfinite(F.d[0]) || !isfinite(F.d[1])) flag = GROUP_NONFINITE;
  else if (F.d[1] == 0. || !isfinite(u) || !(u > 0.)) flag = GROUP_ILL_CONDITIONED;
  group[j] = flag ? NAN : u;
  flags[j] = flag;
}

}  // namespace md200
