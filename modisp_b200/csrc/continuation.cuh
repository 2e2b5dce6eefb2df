// continuation.cuh -- anchor continuation over each model's periods (option
// `continuation`, off by default; the reference's
// frequency_strategy="anchor_continuation": cpp/common/continuation.hpp:12-212,
// cpp/cpu/continuation.hpp:7-36, cpp/cpu/solver.cpp:603-705).
//
// Anchors (every `anchor_stride`-th period, closer where the log step would pass
// 0.25) are solved by the full search.  Every other period is a target: its
// roots are predicted by cubic Hermite interpolation in ln T between the roots
// and slopes dc/dln T of its two anchors, bracketed and refined locally in FP64,
// and audited -- probes on both sides of every root, and the sign and size of
// the function on every gap between brackets (density-spaced points, every body
// velocity +-1e-7, the top-layer Rayleigh/Love and Scholte speeds).  Any doubt
// sends the target to the full FP64 search (PredictionFlag.FALLBACK with the
// reason bits).  Kernels, in launch order:
//   continuation_plan      one thread per model: anchors and targets of its periods
//   anchor_slopes          one thread per anchor root: dc/dln T = c (c/U - 1)
//                          from the forward-mode derivatives, and the anchor's
//                          safety (cpp/common/continuation.hpp:23-31)
//   continuation_predict   one thread per target: Hermite predictions and their
//                          caps (continuation.hpp:33-68), the root work list
//   continuation_root      one thread per predicted root: bracket, refine,
//                          accept test, window probes (continuation.hpp:126-212)
//   continuation_audit     one warp per target: rank order, then the gap audit
//                          32 points at a time (continuation.hpp:70-124); the
//                          verdict (accepted, or the FP64 fallback list)
#pragma once
#include "kernels.cuh"

namespace md200 {

// PredictionFlag bits (python/modisp/__init__.py:55-68)
constexpr unsigned P_ANCHOR = 1u, P_ACCEPTED = 2u, P_FALLBACK = 4u, P_BYPASSED = 8u, P_AUDIT = 16u,
                   P_AUDIT_FAILED = 32u, P_SOURCE_UNCERTAIN = 64u, P_ROOT_COUNT = 128u, P_ANCHOR_UNSAFE = 256u,
                   P_WINDOW = 512u, P_BRACKET = 1024u, P_CORRECTION = 2048u;
constexpr unsigned TRACE_APPROXIMATE_SEARCH = 2048u;
// trace-flag bits that make an anchor's roots unusable as a source
// (TRACE_SEARCH_UNCONVERGED .. F_REJECTED, SAMPLING_UNCERTAIN, ROOT_CONFLICT)
constexpr unsigned SOURCE_UNUSABLE = 4u | 8u | 16u | 32u | 64u | 128u | 512u | 1024u;
// a root code's stage: the rank-order test of a root sits between its refinement
// (stage 1 failures) and its accept test and window probes (stage 2)
constexpr unsigned CODE_STAGE2 = 1u << 31;
constexpr unsigned CODE_AUDITED = 1u << 30;

// ---------------------------------------------------------------------------
// continuation_plan: one thread per model, over the model's own periods (the
// batch's shared periods, or its CSR list in a ragged batch).  A model
// continues when it has at least 8 strictly ascending periods and some target:
// anchors every `stride` periods, closer where the log step would pass 0.25;
// every period between two anchors is a target (cpp/cpu/continuation.hpp:14-27,
// cpp/common/continuation.hpp:17-21).  Roles and anchor traces per trace.
// ---------------------------------------------------------------------------
__global__ void continuation_plan(Dev d, int stride) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= d.B) return;
  int first, T;
  const double *p;
  if (d.ragged) {
    first = d.r_offsets[b];
    T = d.r_offsets[b + 1] - first;
    p = d.periods + first;
  } else {
    first = b * d.T;
    T = d.T;
    p = d.periods;
  }
  bool ok = T >= 8;
  for (int f = 1; f < T && ok; ++f) ok = p[f] > p[f - 1];
  for (int f = 0; f < T; ++f) {
    d.crole[first + f] = 0;
    d.cleft[first + f] = d.cright[first + f] = -1;
  }
  if (!ok) return;
  int targets = 0;
  for (int left = 0;;) {
    d.crole[first + left] = 1;
    if (left == T - 1) break;
    int right = left + (stride < T - 1 - left ? stride : T - 1 - left);
    while (right > left + 1 && log_step(p[right], p[left]) > .25) --right;
    for (int f = left + 1; f < right; ++f) {
      d.crole[first + f] = 2;
      d.cleft[first + f] = first + left;
      d.cright[first + f] = first + right;
      ++targets;
    }
    left = right;
  }
  if (!targets)
    for (int f = 0; f < T; ++f) d.crole[first + f] = 0;
}

// Root i of trace t as assemble left it (ascending, in the slots' root field).
__device__ __forceinline__ double slot_root(const Dev &d, int t, int i) {
  return d.slot[(static_cast<size_t>(t) * d.KB + i) * SLOT + 4];
}
__device__ __forceinline__ double *slot_at(const Dev &d, int t, int i) {
  return d.slot + (static_cast<size_t>(t) * d.KB + i) * SLOT;
}

// ---------------------------------------------------------------------------
// anchor_slopes: one thread per (anchor trace, root).  On the dispersion curve
// F(w / c, w) = 0, dk/dw = -F_w / F_k = 1 / U, so dc/dln T = c (c / U - 1)
// (the reference estimates the same slope by finite differences,
// cpp/common/group_velocity.hpp:94).  The first thread of a trace also decides
// whether its roots can seed predictions.
// ---------------------------------------------------------------------------
__global__ void anchor_slopes(Dev d) {
  const long long q = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (q >= static_cast<long long>(d.n_traces) * d.KB) return;
  const int t = static_cast<int>(q / d.KB), i = static_cast<int>(q - static_cast<long long>(t) * d.KB);
  if (d.crole[t] != 1) return;
  const int b = d.tr_model[t];
  double *slope = d.cslope + static_cast<size_t>(t) * d.KB;
  const int nr = d.ocounts[t], K = d.tr_modes[t] + 2;
  if (i == 0) {
    bool safe = d.mstate[b] == 0 && nr >= 1 && nr <= K && !(d.oflags[t] & SOURCE_UNUSABLE);
    for (int j = 0; j < nr && safe; ++j) {
      const double c = slot_root(d, t, j);
      if (!isfinite(c) || !(c > 0.)) safe = false;
      else if (j && c - slot_root(d, t, j - 1) <= d.close_rtol * c) safe = false;
    }
    d.csafe[t] = safe ? 1 : 0;
    if (d.stats) atomicAdd(&d.stats[17], 1ULL);
  }
  if (d.mstate[b] != 0 || i >= nr || nr > K) {
    slope[i] = NAN;
    return;
  }
  const double c = slot_root(d, t, i), w = TWO_PI / d.tr_period[t];
  using D2 = Dual<double, 2>;
  D2 k, wd;
  k.v = w / c; k.d[0] = 1.; k.d[1] = 0.;
  wd.v = w; wd.d[0] = 0.; wd.d[1] = 1.;
  const D2 F = secular<D2, double>(global_view(d, b), d.wave, k, wd, nullptr);
  const double fk = F.d[0], fw = F.d[1];
  slope[i] = fk != 0. ? c * (-c * fw / fk - 1.) : NAN;
}

// A target's FP64 fallback: the full search, with the prediction verdict.
__device__ __forceinline__ void cont_fallback(const Dev &d, int t, unsigned word) {
  if (d.pred) d.pred[t] = word | P_FALLBACK;
  const int pos = atomicAdd(&d.ctr[C_NREPAIR], 1);
  d.repair_list[pos] = t;
  d.nbr[t] = 0;
  d.tflags[t] = d.fp32 ? TRACE_FP64_REPAIR : 0u;
  if (d.stats) atomicAdd(&d.stats[14], 1ULL);
}

// ---------------------------------------------------------------------------
// continuation_predict: one thread per target (cpp/cpu/solver.cpp:662-679 and
// cpp/common/continuation.hpp:41-68).  Predictions, their disagreement and cap
// go to the target's slots ([0] c, [1] disagreement, [2] cap); each root becomes
// an item of the root list.
// ---------------------------------------------------------------------------
__global__ void continuation_predict(Dev d) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q == 0) restart_lists(d);
  if (q >= *(volatile int *)&d.ctr[C_NTARGET]) return;
  const int t = d.cont_list[q];
  const int b = d.tr_model[t];
  const int tl = d.cleft[t], tr = d.cright[t];
  const int K = d.tr_modes[t] + 2, nr = d.ocounts[tl];
  const unsigned flags = ((d.oflags[tl] | d.oflags[tr]) & TRACE_CLOSE_ROOT_RISK) ? P_SOURCE_UNCERTAIN : 0u;
  unsigned reason = 0;
  if (nr <= 0 || nr > K || d.ocounts[tr] != nr) reason = P_ROOT_COUNT;
  else if (!d.csafe[tl] || !d.csafe[tr]) reason = P_ANCHOR_UNSAFE;
  const double lower = d.mlo[b], upper = d.mhi[b];
  const double pf = d.tr_period[t];
  const double dl = log_step(pf, d.tr_period[tl]), dr = log_step(pf, d.tr_period[tr]);
  if (!reason && !(dl > 0. && dr < 0. && upper > lower)) reason = P_WINDOW;
  if (!reason) {
    const double span = dl - dr, u = dl / span, u2 = u * u, u3 = u2 * u;
    const double *sl = d.cslope + static_cast<size_t>(tl) * d.KB, *sr = d.cslope + static_cast<size_t>(tr) * d.KB;
    double last_left = 0., last_right = 0., last_upper = 0., prev = 0.;
    for (int j = 0; j < nr && !reason; ++j) {
      const double c0 = slot_root(d, tl, j), c1 = slot_root(d, tr, j), s0 = sl[j], s1 = sr[j];
      if (!isfinite(s0) || !isfinite(s1)) { reason = P_ANCHOR_UNSAFE; break; }
      const double cl = c0 + s0 * dl, cr = c1 + s1 * dr;
      const double c = (2. * u3 - 3. * u2 + 1.) * c0 + (u3 - 2. * u2 + u) * span * s0 + (-2. * u3 + 3. * u2) * c1 +
                       (u3 - u2) * span * s1;
      if (!isfinite(c) || !isfinite(cl) || !isfinite(cr) || !(c > lower && c < upper)) { reason = P_WINDOW; break; }
      // the tangent projections from both anchors must keep neighbouring ranks in order
      const double plo = fmin(cl, cr), phi = fmax(cl, cr);
      if (j && (c <= prev || cl <= last_left || cr <= last_right || plo <= last_upper)) {
        reason = P_WINDOW | PRED_REVIEW;
        break;
      }
      last_left = cl; last_right = cr; last_upper = phi; prev = c;
      double *s = slot_at(d, t, j);
      s[0] = c;
      s[1] = fmax(fabs(cl - cr), fabs(c - ((1. - u) * c0 + u * c1)));
    }
    if (!reason) {
      // caps of the local searches (cpp/common/continuation.hpp:33-39, :63-66)
      double *pc = d.slot + static_cast<size_t>(t) * d.KB * SLOT;  // predictions at stride SLOT
      for (int j = 0; j < nr && !reason; ++j) {
        double g = fmin(pc[j * SLOT] - lower, upper - pc[j * SLOT]);
        if (j) g = fmin(g, pc[j * SLOT] - pc[(j - 1) * SLOT]);
        if (j + 1 < nr) g = fmin(g, pc[(j + 1) * SLOT] - pc[j * SLOT]);
        const double cap = fmin(.02 * pc[j * SLOT], .2 * g);
        if (!(cap > 16. * d.tol * pc[j * SLOT]) || pc[j * SLOT + 1] > .5 * cap) reason = P_WINDOW;
        pc[j * SLOT + 2] = cap;
      }
    }
  }
  if (reason) {
    cont_fallback(d, t, flags | reason);
    return;
  }
  if (d.pred) d.pred[t] = flags;  // completed by continuation_audit
  d.nbr[t] = nr;
  const int base = atomicAdd(&d.ctr[C_NCROOT], nr);
  for (int j = 0; j < nr; ++j) d.croot_list[base + j] = t * d.KB + j;
}

// FP64 secular value and shape feature, out of line (one evaluation site for
// the divergent lanes of the continuation kernels).
__device__ __noinline__ double cont_eval(const LayerView<double> m, int wave, double w, double c, double *g) {
  return secular<double, double>(m, wave, w / c, w, g);
}
__device__ __noinline__ RootSample cont_sample(const LayerView<double> m, int wave, double w, double c) {
  return root_sample(m, wave, w, c);
}

// ---------------------------------------------------------------------------
// continuation_root: one thread per predicted root (cpp/common/continuation.hpp:
// 181-211 for one j): widening brackets around the prediction, Brent refinement
// to the run's tolerance, the accept test, and three probes on each open side of
// the root (a same-sign trough among them, which the reference minimises, is
// taken as doubt here).  Writes the bracket and root to the slot and a code.
// ---------------------------------------------------------------------------
__global__ void continuation_root(Dev d) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= *(volatile int *)&d.ctr[C_NCROOT]) return;
  const int id = d.croot_list[i];
  const int t = id / d.KB, j = id - t * d.KB;
  const int b = d.tr_model[t];
  const int tl = d.cleft[t], tr = d.cright[t];
  const double lower = d.mlo[b], upper = d.mhi[b], tol = d.tol;
  const double pf = d.tr_period[t], w = TWO_PI / pf;
  const double dl = log_step(pf, d.tr_period[tl]), dr = log_step(pf, d.tr_period[tr]);
  const LayerView<double> m = global_view(d, b);
  double *s = slot_at(d, t, j);
  const double c = s[0], disagreement = s[1], cap = s[2];
  unsigned long long evals = 0;
  unsigned code = 0;
  double width = fmin(cap, fmax(16. * tol * c, fmax(2. * disagreement, .05 * c * fmin(fabs(dl), fabs(dr)))));
  double a = 0., bb = 0., fa = 0., fb = 0., g;
  bool bracket = false;
  for (int attempt = 0; attempt < 4; ++attempt) {
    a = fmax(lower, c - width);
    bb = fmin(upper, c + width);
    fa = cont_eval(m, d.wave, w, a, &g);
    fb = cont_eval(m, d.wave, w, bb, &g);
    evals += 2;
    if (isfinite(fa) && isfinite(fb) && fa != 0. && fb != 0. && ((fa < 0.) != (fb < 0.))) {
      bracket = true;
      break;
    }
    if (width >= cap) break;
    width = fmin(cap, 2. * width);
  }
  double root = NAN;
  if (!bracket) {
    code = P_BRACKET;
  } else {
    BrentState st;
    brent_init(st, a, bb, fa, fb);
    for (int it = 0; it <= BRENT_MAX_EVALS; ++it) {
      double x;
      const int r = brent_advance(st, tol, &x, &root);
      if (r != BRENT_EVAL) {
        if (r != BRENT_DONE) root = NAN;
        break;
      }
      brent_absorb(st, cont_sample(m, d.wave, w, x));
      ++evals;
    }
    if (!isfinite(root) || root < a || root > bb) code = P_CORRECTION;
  }
  if (!code && d.accept < 1.) {
    const double v = cont_eval(m, d.wave, w, root, &g);
    ++evals;
    if (!isfinite(v) || fabs(v) > d.accept) code = CODE_STAGE2 | P_CORRECTION;
  }
  if (!code) {
    // probes on both open sides of the root, outside its numerical uncertainty
    const double margin = fmax(tol, 16. * 2.220446049250313e-16) * root;
    for (int side = 0; side < 2 && !code; ++side) {
      const double edge = side ? bb : a, sign = (side ? fb : fa) < 0. ? -1. : 1.;
      if (fabs(root - edge) <= 2. * margin) continue;
      const double end = root + copysign(margin, edge - root), step = (end - edge) * .25;
      double mag[3] = {0., 0., 0.};
      for (int k = 0; k < 3 && !code; ++k) {
        const double v = cont_eval(m, d.wave, w, edge + (k + 1) * step, &g);
        ++evals;
        if (!isfinite(v) || !isfinite(g)) code = CODE_STAGE2 | CODE_AUDITED | P_AUDIT_FAILED;
        else if (sign * v <= 0.) code = CODE_STAGE2 | CODE_AUDITED | P_AUDIT_FAILED | PRED_REVIEW;
        mag[k] = sign * g;
      }
      if (!code && mag[1] < mag[0] && mag[1] < mag[2] && (mag[1] < .5 * fmin(mag[0], mag[2]) || mag[1] < .05))
        code = CODE_STAGE2 | CODE_AUDITED | P_AUDIT_FAILED | PRED_REVIEW;
    }
  }
  s[0] = a;
  s[1] = bb;
  s[2] = fa;
  s[3] = fb;
  s[4] = root;
  d.ccode[id] = code;
  if (d.stats) {
    atomicAdd(&d.stats[0], evals);
    atomicAdd(&d.stats[2], evals * static_cast<unsigned long long>(layer_steps(m.L, m.water)));
    atomicAdd(&d.stats[18], evals);
  }
}

// Inverse of the phase-count density N(c) (cpp/common/physics.hpp:180-193):
// the knot table brackets the target, regula falsi with bisection every fourth
// step closes it.
__device__ double inverse_count(const Dev &d, int b, double target) {
  const double4 *kt = d.knot + static_cast<size_t>(b) * d.nkmax;
  const int nk = d.nknot[b];
  int lo = 0, hi = nk - 1;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (kt[mid].y < target) lo = mid; else hi = mid;
  }
  double a = kt[lo].x, bb = kt[hi].x, fa = kt[lo].y, fb = kt[hi].y;
  const double *tab = layer_table<double>(d, b);
  const double eps = 1e-9 * fmax(1., fabs(target));
  double x = .5 * (a + bb);
  for (int it = 0; it < 48; ++it) {
    x = a + (bb - a) * (target - fa) / (fb - fa);
    if (it % 4 == 3 || !isfinite(x) || x <= a || x >= bb) x = .5 * (a + bb);
    const double v = phase_count(tab, d.Ls, d.mL[b], d.wave, x);
    if (fabs(v - target) <= eps || bb - a <= 8e-15 * fmax(1., fabs(x))) return x;
    if (v < target) { a = x; fa = v; } else { bb = x; fb = v; }
  }
  return .5 * (a + bb);
}

// ---------------------------------------------------------------------------
// continuation_audit: one warp per target that was predicted (128-thread
// blocks).  Root codes in rank order (with the rank-order test between
// refinement and the stage-2 checks), then the gap audit
// (cpp/common/continuation.hpp:85-124): the sign at both ends of every gap, then
// its midpoint, the density-spaced points, every body velocity +-1e-7 and the
// model's two seed speeds inside it, 32 points per warp step.  The verdict:
// accepted (roots in the slots, TRACE_APPROXIMATE_SEARCH |
// CONTINUATION_APPROXIMATE) or the FP64 fallback.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) continuation_audit(Dev d) {
  __shared__ double gsign[4][64], gmin[4][64];  // the gaps of each warp, 64 at a time
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int warps = (gridDim.x * blockDim.x) >> 5, wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int ntarget = *(volatile int *)&d.ctr[C_NTARGET];
  unsigned long long evals = 0;
  for (int q = wid; q < ntarget; q += warps) {
    const int t = d.cont_list[q];
    if (d.nbr[t] == 0) continue;  // sent to the fallback by continuation_predict
    const int b = d.tr_model[t];
    const int K = d.tr_modes[t] + 2, nr = d.nbr[t];
    const double lower = d.mlo[b];
    const double w = TWO_PI / d.tr_period[t];
    const LayerView<double> m = global_view(d, b);
    const double *sl = d.slot + static_cast<size_t>(t) * d.KB * SLOT;
    // 1. root codes in rank order: the first failing root decides
    unsigned reason = 0;
    bool audited = false;
    for (int base = 0; base < nr; base += 32) {
      const int j = base + lane;
      unsigned code = 0;
      if (j < nr) {
        const unsigned raw = d.ccode[t * d.KB + j];
        if (raw && !(raw & CODE_STAGE2)) code = raw;
        if (!code && j) {
          const double r = sl[j * SLOT + 4], p = sl[(j - 1) * SLOT + 4];
          if (r - p <= d.close_rtol * fabs(r) || (d.fp32 && static_cast<float>(r) <= static_cast<float>(p)))
            code = P_CORRECTION | PRED_REVIEW;
        }
        if (!code) code = raw & ~CODE_STAGE2;
      }
      const unsigned fm = __ballot_sync(FULL, code != 0);
      if (fm) {
        const unsigned c = __shfl_sync(FULL, code, __ffs(fm) - 1);
        audited = (c & CODE_AUDITED) != 0;  // the window probes of that root ran
        reason = c & ~CODE_AUDITED;
        break;
      }
    }
    // 2. the gap audit
    if (!reason) {
      audited = true;
      const double upper = nr == K ? sl[(nr - 1) * SLOT + 1] : d.mhi[b];
      const int G = nr + (nr < K ? 1 : 0);
      // gap g spans (a_g, b_g): a_g = hi of bracket g-1 (or lower), b_g = lo of bracket g (or upper)
      auto gap_a = [&](int gi) { return gi ? sl[(gi - 1) * SLOT + 1] : lower; };
      auto gap_b = [&](int gi) { return gi < nr ? sl[gi * SLOT] : upper; };
      const double *tab = layer_table<double>(d, b);
      const int L = m.L, top = m.water;
      const double nlo = phase_count(tab, d.Ls, L, d.wave, lower), nhi = phase_count(tab, d.Ls, L, d.wave, upper);
      double seeds[2] = {NAN, NAN};
      {
        const double vp0 = tab[7 * d.Ls + top], vs0 = tab[8 * d.Ls + top];
        seeds[0] = d.wave ? vs0 : rayleigh_speed(vp0, vs0);
        if (!d.wave && top)
          seeds[1] = scholte_speed(tab[7 * d.Ls], tab[4 * d.Ls], tab[7 * d.Ls + 1], tab[8 * d.Ls + 1], tab[4 * d.Ls + 1]);
      }
      unsigned fail = 0;
      for (int gb = 0; gb < G && !fail; gb += 64) {
        // ends of every gap: their sign and the smaller shape magnitude
        int fail_gap = 1 << 30;
        for (int gi = gb + lane; gi < gb + 64; gi += 32) {
          double sa = 0., ma = INFINITY;
          if (gi < G) {
            const double a = gap_a(gi), bb = gap_b(gi);
            if (bb > a) {
              double ga, gbv;
              const double fa = cont_eval(m, d.wave, w, a, &ga), fb = cont_eval(m, d.wave, w, bb, &gbv);
              evals += 2;
              unsigned bad = 0;
              if (!isfinite(fa) || !isfinite(fb) || !isfinite(ga) || !isfinite(gbv)) bad = P_AUDIT_FAILED;
              else if (fa == 0. || fb == 0.)
                bad = ((fa == 0. && a > lower) || (fb == 0. && bb < upper)) ? P_AUDIT_FAILED | PRED_REVIEW
                                                                           : P_AUDIT_FAILED;
              else if ((fa < 0.) != (fb < 0.)) bad = P_AUDIT_FAILED | PRED_REVIEW;
              if (bad && gi < fail_gap) { fail_gap = gi; fail = bad; }
              sa = fa < 0. ? -1. : 1.;
              ma = fmin(fabs(ga), fabs(gbv));
            }
          }
          gsign[wib][gi - gb] = sa;
          gmin[wib][gi - gb] = ma;
        }
        for (int o = 16; o; o >>= 1) {  // the earliest failing gap decides
          const int og = __shfl_xor_sync(FULL, fail_gap, o);
          const unsigned of = __shfl_xor_sync(FULL, fail, o);
          if (og < fail_gap) { fail_gap = og; fail = of; }
        }
        __syncwarp();
        if (fail) break;
        // interior points: midpoints of these gaps, density points, body velocities
        // +-1e-7, seeds -- each tested against the gap it lies in
        const int npts = 64 + 31 + 6 * L + 2;
        for (int p0 = 0; p0 < npts && !fail; p0 += 32) {
          const int p = p0 + lane;
          double c = NAN;
          if (p < 64) {
            const int gi = gb + p;
            if (gi < G) c = gap_a(gi) + .5 * (gap_b(gi) - gap_a(gi));
          } else if (p < 64 + 31) {
            const double target = nlo + (nhi - nlo) * (p - 63) / 32.;
            c = nhi > nlo ? inverse_count(d, b, target) : lower + (upper - lower) * (p - 63) / 32.;
          } else if (p < 64 + 31 + 6 * L) {
            const int q6 = p - 64 - 31, layer = q6 / 6, r6 = q6 - layer * 6;
            if (!(d.wave && top && layer == 0)) {
              const double v = r6 < 3 ? tab[7 * d.Ls + layer] : tab[8 * d.Ls + layer];
              c = v * (1. + (r6 % 3 - 1) * 1e-7);
            }
          } else if (p < npts) {
            c = seeds[p - 64 - 31 - 6 * L];
          }
          int gi = -1;  // the gap (among gb .. gb+63) that holds c
          if (isfinite(c))
            for (int x = gb; x < gb + 64 && x < G; ++x)
              if (c > gap_a(x) && c < gap_b(x)) { gi = x; break; }
          unsigned bad = 0;
          if (gi >= 0 && gsign[wib][gi - gb] != 0.) {
            double gv;
            const double v = cont_eval(m, d.wave, w, c, &gv);
            ++evals;
            const double sg = gsign[wib][gi - gb];
            if (!isfinite(v) || !isfinite(gv)) bad = P_AUDIT_FAILED;
            else if (v == 0. || (v < 0.) != (sg < 0.) || (fabs(gv) < .05 && fabs(gv) < .1 * gmin[wib][gi - gb]))
              bad = P_AUDIT_FAILED | PRED_REVIEW;
          }
          int fg = bad ? gi : 1 << 30;
          unsigned fv = bad;
          for (int o = 16; o; o >>= 1) {
            const int og = __shfl_xor_sync(FULL, fg, o);
            const unsigned of = __shfl_xor_sync(FULL, fv, o);
            if (og < fg) { fg = og; fv = of; }
          }
          if (fv) fail = fv;
        }
        __syncwarp();
      }
      reason = fail;
    }
    if (lane == 0) {
      const unsigned word = (d.pred ? d.pred[t] : 0u) | (audited ? P_AUDIT : 0u);
      if (reason) {
        cont_fallback(d, t, word | reason);
      } else {
        if (d.pred) d.pred[t] = word | P_ACCEPTED;
        d.tflags[t] = TRACE_APPROXIMATE_SEARCH | TRACE_CONTINUATION_APPROXIMATE;
        if (d.stats) atomicAdd(&d.stats[13], 1ULL);
      }
    }
    __syncwarp();
  }
  if (d.stats && evals) {
    atomicAdd(&d.stats[0], evals);
    atomicAdd(&d.stats[18], evals);
  }
}

}  // namespace md200
