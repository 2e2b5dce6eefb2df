// uniform.cuh -- the legacy uniform-grid Rayleigh path: the reference's
// search_strategy="uniform" (python/modisp/_legacy.py:124-431 over
// cpp/cuda/coarse_scan.cuh:19-70 and cpp/cuda/refine.cuh:33-317), solid models.
//
// Stage 1 samples F in single precision on the grid c_i = cmin + i dc,
// i = 0..nc-1, dc = (cmax - cmin) / (nc - 1), per (model, period); stage 2 walks
// each row in order: a sign change between cells i and i+1 is the next mode; a
// strict point trough of |F| below 0.05 between two sign-free cells is
// sub-sampled in FP64 at 66 points, each sign change there being the next
// (hidden) mode.  Each mode's bracket is confirmed in FP64 (a rejected cell is
// replaced by an adjacent sign-free cell whose FP64 ends differ in sign, when
// exactly one of the two does), bisected a fixed number of times, optionally
// screened by |F(root)| and dropped at or above the half-space shear velocity.
//
// B200 form, four kernels:
//   uniform_prep    warp per model: the engine's FP64/FP32 layer tables
//                   (zero-thickness rows, identity steps, dropped)
//   uniform_scan    warp per 32 consecutive cells of one row: FP32 values on the
//                   max-amplitude scale of the reference's normalised recurrence
//   uniform_walk    warp per row: the row's events classified 32 cells at a time
//                   (ballots), troughs sub-sampled by the whole warp, one bracket
//                   record per found mode and the records' indices appended to a
//                   work list
//   uniform_bisect  thread per listed bracket: confirmation, relocation,
//                   bisection, acceptance -- the FP64 work, with no idle lanes
//                   for modes a row does not have
// The reference runs stage 2 as one thread per (model, period, mode), each
// re-walking its row from the start and sub-sampling every trough before its
// mode.  The events, their order and every bracket are the same here; the
// statistics are counted as the reference's threads count them (a trough counts
// once for every mode thread that passes it).
#pragma once
#include "kernels.cuh"

namespace md200 {

constexpr int UNIFORM_SUBSAMPLES = 64;          // interior samples of a trough window
constexpr float UNIFORM_TROUGH_MAX_ABS = 0.05f;  // |F| a point trough must fall below
constexpr unsigned UNIFORM_UNRESOLVED = 1u, UNIFORM_RELOCATED = 2u;  // trace flags
enum UniformStat {
  US_BRACKETS = 0,  // sign-change brackets bisected
  US_REJECTED_SIGN, // FP64 did not confirm the FP32 sign change
  US_REJECTED_F,    // |F(root)| above f_accept
  US_TROUGHS,       // troughs passed, once per mode thread that passes them
  US_HIDDEN,        // roots recovered by sub-sampling
  US_RELOCATED,     // rejected brackets recovered from a neighbouring cell
  US_COUNT
};

// One mode's bracket: a sign-change cell (cell >= 0; its ends are grid points)
// or a sub-sampled one (cell = -1: lo, hi and the FP64 value at lo).
struct UniformBracket {
  double lo, hi, flo;
  int cell, pad;
};

struct UniformDev {
  int B, Lmax, Ls, nf, nc, K;
  const double *h, *vp, *vs, *rho;  // inputs [B][Lmax]
  double *layer64;                  // [B][ROWS][Ls]
  float *layer32;                   // [B][ROWS][Ls]
  int *mL;                          // rows kept per model
  const float *periods;             // [nf], single precision as the reference stores them
  const float *rows;                // stage 1 values [B][nf][nc]
  double *out;                      // [B][K][nf]
  unsigned *flags;                  // [B][nf]
  unsigned long long *stats;        // [US_COUNT]
  UniformBracket *br;               // [B * nf][K]
  int *list, *count;                // indices into br of found modes
};

// grid point i in FP64 (cpp/cuda/refine.cuh:33-35: cmin + dc * i, one rounding)
__device__ __forceinline__ double uniform_c(double cmin, double dc, int i) {
  return __fma_rn(dc, static_cast<double>(i), cmin);
}

// Highest grid index stage 2 reads as a cell start (cpp/common/scan_grid.hpp:19-24):
// the half-space shear velocity caps the trapped-mode domain.
__device__ __forceinline__ int uniform_i_last(double c_cap, double cmin, double dc, int nc) {
  int i = static_cast<int>((c_cap - cmin) / dc);
  if (i > nc - 2) i = nc - 2;
  return i;
}

__device__ __forceinline__ double uniform_vs_half_space(const UniformDev &u, int b) {
  return u.layer64[static_cast<size_t>(b) * ROWS * u.Ls + 8 * u.Ls + u.mL[b] - 1];
}

// F at velocity c, angular frequency w, in FP64: wavenumber w / c from the
// caller's w, the recurrence with w clamped at 1e-4 (cpp/common/dunkin.hpp:365).
// `fmax`: the value on the max-amplitude scale.
__device__ __forceinline__ double uniform_f64(const LayerView<double> &m, double w, double c,
                                              double *fmax = nullptr) {
  const double k = w / c, wc = w < 1e-4 ? 1e-4 : w;
  double F;
  rayleigh_multi<double, double, 1>(m, &k, wc, &F, nullptr, nullptr, nullptr, fmax);
  return F;
}

// ---------------------------------------------------------------------------
// uniform_prep: one warp per model, the engine's table layout (prep_models'
// first step): rows h (0 for the half-space), 1/vp, 1/vs, vs^2, rho, 1/rho,
// 1/(rho vs^2), vp, vs; row 0, the half-space and every layer of positive
// thickness kept.
// ---------------------------------------------------------------------------
__global__ void uniform_prep(UniformDev u) {
  const int lane = threadIdx.x & 31;
  const int b = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (b >= u.B) return;
  const size_t in = static_cast<size_t>(b) * u.Lmax;
  double *t64 = u.layer64 + static_cast<size_t>(b) * ROWS * u.Ls;
  float *t32 = u.layer32 + static_cast<size_t>(b) * ROWS * u.Ls;
  int L = 0;
  for (int base = 0; base < u.Lmax; base += 32) {
    const int j = base + lane;
    bool keep = false;
    double hj = 0., vpj = 1., vsj = 1., rj = 1.;
    if (j < u.Lmax) {
      hj = u.h[in + j];
      vpj = u.vp[in + j];
      vsj = u.vs[in + j];
      rj = u.rho[in + j];
      keep = j == 0 || j == u.Lmax - 1 || hj > 0.;
    }
    const unsigned mask = __ballot_sync(FULL, keep);
    if (keep) {
      const int r = L + __popc(mask & lanemask_lt());
      const double vals[ROWS] = {j == u.Lmax - 1 ? 0. : hj, 1. / vpj, 1. / vsj, vsj * vsj, rj, 1. / rj,
                                 1. / (rj * vsj * vsj), vpj, vsj};
#pragma unroll
      for (int q = 0; q < ROWS; ++q) {
        t64[q * u.Ls + r] = vals[q];
        t32[q * u.Ls + r] = static_cast<float>(vals[q]);
      }
    }
    L += __popc(mask);
  }
  if (lane == 0) u.mL[b] = L;
}

// ---------------------------------------------------------------------------
// uniform_scan: stage 1 (cpp/cuda/coarse_scan.cuh:19-70).  One warp per 32
// consecutive cells of one (model, period) row: the warp shares its model and
// period.  Cells past the last one stage 2 reads hold NaN.  The grid point is
// formed in FP64 and rounded to single precision; w = 2 pi / T and k = w / c
// are correctly rounded single-precision quotients, as the reference's
// default-precision build computes them.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) uniform_scan(UniformDev u, float *rows, double cmin, double dc) {
  const int lane = threadIdx.x & 31;
  const int nch = (u.nc + 31) >> 5;
  const long long units = static_cast<long long>(u.B) * u.nf * nch;
  const long long stride = static_cast<long long>(gridDim.x) * (blockDim.x >> 5);
  for (long long wu = static_cast<long long>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); wu < units;
       wu += stride) {
    const long long row = wu / nch;
    const int ic = static_cast<int>(wu - row * nch) * 32 + lane;
    const int f = static_cast<int>(row % u.nf), b = static_cast<int>(row / u.nf);
    if (ic >= u.nc) continue;
    const int last = uniform_i_last(uniform_vs_half_space(u, b), cmin, dc, u.nc) + 1;
    float v = NAN;
    if (ic <= last) {
      const LayerView<float> m =
          make_view<float>(u.layer32 + static_cast<size_t>(b) * ROWS * u.Ls, u.Ls, u.mL[b], 0);
      const float w = __fdiv_rn(6.283185307179586f, u.periods[f]);
      const float c = static_cast<float>(uniform_c(cmin, dc, ic));
      const float k = __fdiv_rn(w, c);
      float F, fm;
      rayleigh_multi<float, float, 1>(m, &k, w < 1e-4f ? 1e-4f : w, &F, nullptr, nullptr, nullptr, &fm);
      v = fm;
    }
    rows[row * u.nc + ic] = v;
  }
}

// ---------------------------------------------------------------------------
// uniform_walk: stage 2's row walk (cpp/cuda/refine.cuh:175-245), one warp per
// (model, period) row, 32 cells classified at a time:
//   sign change   (F_i < 0) != (F_i+1 < 0), i <= i_last;
//   point trough  at i+1 after a sign-free cell i: cell (i+1, i+2) sign-free,
//                 |F_i| > |F_i+1| < |F_i+2|, |F_i+1| < 0.05, i+1 <= i_last.
// The reference's walk resumes two cells on after a trough window [i, i+2];
// the cell it skips is sign-free and cannot start a trough (strict minima are
// never adjacent), so classifying every cell yields its events in its order.
// A trough window is sub-sampled by the warp: samples j = 0..65 at
// c_i + (span j) / 65 (three per lane at most), each sign change between
// samples j-1 and j the next mode.  The walk ends at the K-th mode; the
// records of the found modes go to the work list, missing modes are NaN.
// Troughs are counted as the reference's mode threads count them: once for
// each mode whose walk passes the trough (the walk of a mode the row does not
// have passes all of them).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128, 4) uniform_walk(UniformDev u, double cmin, double dc) {
  const int lane = threadIdx.x & 31;
  const long long nrow = static_cast<long long>(u.B) * u.nf;
  const long long stride = static_cast<long long>(gridDim.x) * (blockDim.x >> 5);
  unsigned long long passes = 0;
  for (long long t = static_cast<long long>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); t < nrow;
       t += stride) {
    const int f = static_cast<int>(t % u.nf), b = static_cast<int>(t / u.nf);
    const int nc = u.nc, K = u.K;
    const float *row = u.rows + t * nc;
    const int i_last = uniform_i_last(uniform_vs_half_space(u, b), cmin, dc, nc);
    const LayerView<double> m =
        make_view<double>(u.layer64 + static_cast<size_t>(b) * ROWS * u.Ls, u.Ls, u.mL[b], 0);
    const double w = TWO_PI / static_cast<double>(u.periods[f]);
    UniformBracket *br = u.br + t * K;
    int mode = 0, ntr = 0;
    for (int base = 0; base <= i_last && mode < K; base += 32) {
      const int i = base + lane;
      const bool valid = i <= i_last;
      float r0 = 0.f, r1 = 0.f, r2 = 0.f;
      if (valid) {
        r0 = row[i];
        r1 = row[i + 1];
        if (i + 2 < nc) r2 = row[i + 2];
      }
      const bool sc = valid && ((r0 < 0.f) != (r1 < 0.f));
      const bool tr = valid && !sc && i + 1 <= i_last && i + 2 < nc && ((r1 < 0.f) == (r2 < 0.f)) &&
                      fabsf(r0) > fabsf(r1) && fabsf(r1) < fabsf(r2) && fabsf(r1) < UNIFORM_TROUGH_MAX_ABS;
      const unsigned msc = __ballot_sync(FULL, sc);
      unsigned ev = msc | __ballot_sync(FULL, tr);
      while (ev && mode < K) {
        const int l = __ffs(ev) - 1;
        ev &= ev - 1;
        if ((msc >> l) & 1u) {
          if (lane == 0) br[mode] = UniformBracket{0., 0., 0., base + l, 0};
          passes += ntr;
          ++mode;
          continue;
        }
        ++ntr;
        const double ca = uniform_c(cmin, dc, base + l), span = uniform_c(cmin, dc, base + l + 2) - ca;
        double x[3], fv[3], xp[3], fp[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          const int j = lane + 32 * q;
          x[q] = j == 0 ? ca : __dadd_rn(ca, __ddiv_rn(__dmul_rn(span, static_cast<double>(j)),
                                                        static_cast<double>(UNIFORM_SUBSAMPLES + 1)));
          fv[q] = j <= UNIFORM_SUBSAMPLES + 1 ? uniform_f64(m, w, x[q]) : 0.;
        }
#pragma unroll
        for (int q = 0; q < 3; ++q) {  // sample j - 1 beside sample j
          fp[q] = __shfl_up_sync(FULL, fv[q], 1);
          xp[q] = __shfl_up_sync(FULL, x[q], 1);
          const double f31 = __shfl_sync(FULL, fv[q ? q - 1 : 0], 31), x31 = __shfl_sync(FULL, x[q ? q - 1 : 0], 31);
          if (lane == 0) {
            fp[q] = f31;
            xp[q] = x31;
          }
        }
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          const int j = lane + 32 * q;
          unsigned hid = __ballot_sync(FULL, j >= 1 && j <= UNIFORM_SUBSAMPLES + 1 && ((fp[q] < 0.) != (fv[q] < 0.)));
          while (hid && mode < K) {
            const int s = __ffs(hid) - 1;
            hid &= hid - 1;
            const double lo = __shfl_sync(FULL, xp[q], s), hi = __shfl_sync(FULL, x[q], s);
            const double flo = __shfl_sync(FULL, fp[q], s);
            if (lane == 0) br[mode] = UniformBracket{lo, hi, flo, -1, 0};
            passes += ntr;
            ++mode;
          }
        }
      }
    }
    passes += static_cast<unsigned long long>(K - mode) * ntr;
    int first = 0;
    if (lane == 0 && mode) first = atomicAdd(u.count, mode);
    first = __shfl_sync(FULL, first, 0);
    for (int j = lane; j < K; j += 32) {
      if (j < mode) u.list[first + j] = static_cast<int>(t * K + j);
      else u.out[(static_cast<size_t>(b) * K + j) * u.nf + f] = NAN;
    }
  }
  if (lane == 0 && passes) atomicAdd(&u.stats[US_TROUGHS], passes);
}

// The adjacent cell c2 as a replacement for a rejected bracket
// (cpp/cuda/refine.cuh:63-80): its FP64 ends must differ in sign.
__device__ __forceinline__ bool uniform_retry(const LayerView<double> &m, double w, double cmin, double dc,
                                              int c2, int i_last, double &lo, double &hi, double &flo) {
  if (c2 < 0 || c2 > i_last) return false;
  const double a = uniform_c(cmin, dc, c2), b = uniform_c(cmin, dc, c2 + 1);
  const double fa = uniform_f64(m, w, a), fb = uniform_f64(m, w, b);
  if ((fa < 0.) == (fb < 0.)) return false;
  lo = a;
  hi = b;
  flo = fa;
  return true;
}

// ---------------------------------------------------------------------------
// uniform_bisect: stage 2's per-mode work (cpp/cuda/refine.cuh:247-316,
// bisect_store :83-116), one thread per listed bracket.  A sign-change cell is
// confirmed in FP64; a rejected one is replaced by the left or right sign-free
// neighbour whose FP64 ends differ in sign when exactly one does (RELOCATED),
// else the mode is NaN (UNRESOLVED).  Bisection keeps the end whose FP64 sign
// matches the lower end's, `iters` times (one count for every bracket, so the
// warp's lanes stay in step), and returns the midpoint; with f_accept < 1 a root
// whose |F| on the max-amplitude scale exceeds it is NaN.  A root at or above
// the half-space shear velocity is dropped.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128, 4) uniform_bisect(UniformDev u, double cmin, double dc, int iters,
                                                      double f_accept) {
  const int n = *u.count;
  unsigned long long st[US_COUNT] = {};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int id = u.list[i];
    const long long t = id / u.K;
    const int mode = static_cast<int>(id - t * u.K);
    const int f = static_cast<int>(t % u.nf), b = static_cast<int>(t / u.nf);
    const UniformBracket r = u.br[id];
    const LayerView<double> m =
        make_view<double>(u.layer64 + static_cast<size_t>(b) * ROWS * u.Ls, u.Ls, u.mL[b], 0);
    const double w = TWO_PI / static_cast<double>(u.periods[f]);
    const double c_cap = uniform_vs_half_space(u, b);
    double lo = r.lo, hi = r.hi, flo = r.flo;
    bool bracketed = true;
    if (r.cell >= 0) {
      ++st[US_BRACKETS];
      lo = uniform_c(cmin, dc, r.cell);
      hi = uniform_c(cmin, dc, r.cell + 1);
      flo = uniform_f64(m, w, lo);
      const double fhi = uniform_f64(m, w, hi);
      if ((flo < 0.) == (fhi < 0.)) {
        ++st[US_REJECTED_SIGN];
        const float *row = u.rows + t * u.nc;
        const int i_last = uniform_i_last(c_cap, cmin, dc, u.nc);
        const int cl = r.cell - 1, cr = r.cell + 1;
        const bool cand_l = cl >= 0 && ((row[cl] < 0.f) == (row[cl + 1] < 0.f));
        const bool cand_r = cr + 1 < u.nc && cr <= i_last && ((row[cr] < 0.f) == (row[cr + 1] < 0.f));
        double llo = 0., lhi = 0., lflo = 0., rlo = 0., rhi = 0., rflo = 0.;
        const bool left = cand_l && uniform_retry(m, w, cmin, dc, cl, i_last, llo, lhi, lflo);
        const bool right = cand_r && uniform_retry(m, w, cmin, dc, cr, i_last, rlo, rhi, rflo);
        if (left != right) {
          ++st[US_RELOCATED];
          atomicOr(u.flags + t, UNIFORM_RELOCATED);
          lo = left ? llo : rlo;
          hi = left ? lhi : rhi;
          flo = left ? lflo : rflo;
        } else {
          atomicOr(u.flags + t, UNIFORM_UNRESOLVED);
          bracketed = false;
        }
      }
    } else {
      ++st[US_HIDDEN];
    }
    double root = NAN;
    if (bracketed) {
      for (int k = 0; k < iters; ++k) {
        const double mid = 0.5 * (lo + hi);
        const double fm = uniform_f64(m, w, mid);
        if ((fm < 0.) == (flo < 0.)) {
          lo = mid;
          flo = fm;
        } else {
          hi = mid;
        }
      }
      root = 0.5 * (lo + hi);
      if (f_accept < 1.) {
        double fr;
        uniform_f64(m, w, root, &fr);
        if (fabs(fr) > f_accept) {
          root = NAN;
          ++st[US_REJECTED_F];
        }
      }
    }
    if (root == root && root >= c_cap) root = NAN;
    u.out[(static_cast<size_t>(b) * u.K + mode) * u.nf + f] = root;
  }
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int s = 0; s < US_COUNT; ++s) {
    unsigned long long v = st[s];
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    if (lane == 0 && v && s != US_TROUGHS) atomicAdd(&u.stats[s], v);
  }
}

}  // namespace md200
