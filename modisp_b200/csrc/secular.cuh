// secular.cuh -- device secular functions of the modisp_b200 engine.
//
// Rayleigh (P-SV): normalized Dunkin compound-matrix recurrence, the algebra of
//   cpp/common/dunkin.hpp:82-159 (layer eigenfunction products),
//   :171-221 (compound matrix) and :358-448 (half-space start, upward sweep,
//   water top).  The 25 matrix entries are formed from their 15 distinct values
//   and contracted directly with the 5-vector (same matrix, no storage).
// Love (SH): 2-vector Thomson-Haskell recurrence of cpp/common/physics.hpp:33-53.
//
// Everything is generic over the number type N so one source serves the FP32
// scan (N = float), the FP64 scan and refinement (N = double) and the
// forward-mode derivatives used for group velocity and Jacobians
// (N = Dual<double, ND>).  Branches test the value part only, and the per-layer
// normalisation divides by a power of two taken from the value part: the sign
// of F and every root are those of the reference function, and derivative parts
// are the exact derivatives of the unnormalised function times the same positive
// scale (so ratios of derivatives at a root are exact).
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <type_traits>

// Device code by default; MD200_HOST_SECULAR builds the same recurrences for the
// host (with libm in place of the device intrinsics) for CPU-side studies.
#ifdef MD200_HOST_SECULAR
#define MD200_FN __host__ __device__ __forceinline__
#else
#define MD200_FN __device__ __forceinline__
#endif

namespace md200 {

// ---------------------------------------------------------------------------
// Number-type helpers
// ---------------------------------------------------------------------------
// Forward-mode number: value and ND directional derivatives.  T may itself be a
// Dual (nested forward mode: second derivatives, or parameter derivatives of
// the (k, omega) derivatives used by the adjoint Jacobians).
template <class T, int ND>
struct Dual {
  T v;
  T d[ND];
  Dual() = default;
  // a constant of this number type (all derivative parts zero)
  template <class S, typename std::enable_if<std::is_arithmetic<S>::value, int>::type = 0>
  MD200_FN explicit Dual(S x) : v(x) {
#pragma unroll
    for (int i = 0; i < ND; ++i) d[i] = T(0);
  }
};

// Value part of a number (the innermost scalar for nested duals).
MD200_FN double val(double x) { return x; }
MD200_FN float val(float x) { return x; }
template <class T, int ND>
MD200_FN auto val(const Dual<T, ND> &x) { return val(x.v); }

template <class T>
struct Base { using type = T; };
template <class T, int ND>
struct Base<Dual<T, ND>> { using type = typename Base<T>::type; };

template <class T> struct IsDual : std::false_type {};
template <class T, int ND> struct IsDual<Dual<T, ND>> : std::true_type {};

// Constants of the number type.
template <class N> struct Lift;
template <> struct Lift<double> {
  MD200_FN static double one() { return 1.0; }
  MD200_FN static double zero() { return 0.0; }
};
template <> struct Lift<float> {
  MD200_FN static float one() { return 1.0f; }
  MD200_FN static float zero() { return 0.0f; }
};
template <class T, int ND> struct Lift<Dual<T, ND>> {
  MD200_FN static Dual<T, ND> one() { return Dual<T, ND>(1); }
  MD200_FN static Dual<T, ND> zero() { return Dual<T, ND>(0); }
};
template <class N> MD200_FN N lift_one() { return Lift<N>::one(); }
template <class N> MD200_FN N lift_zero() { return Lift<N>::zero(); }

// a * b + c: one rounding for the scalar types, the dual product otherwise
MD200_FN double mul_add(double a, double b, double c) { return ::fma(a, b, c); }
MD200_FN float mul_add(float a, float b, float c) { return fmaf(a, b, c); }
template <class T, int ND>
MD200_FN Dual<T, ND> mul_add(const Dual<T, ND> &a, const Dual<T, ND> &b, const Dual<T, ND> &c);

#define MD200_DUAL_BINOP(OP, VALUE, DERIV)                                              \
  template <class T, int ND>                                                            \
  MD200_FN Dual<T, ND> operator OP(const Dual<T, ND> &a,              \
                                                     const Dual<T, ND> &b) {            \
    Dual<T, ND> r;                                                                      \
    r.v = VALUE;                                                                        \
    _Pragma("unroll") for (int i = 0; i < ND; ++i) r.d[i] = DERIV;                      \
    return r;                                                                           \
  }
MD200_DUAL_BINOP(+, a.v + b.v, a.d[i] + b.d[i])
MD200_DUAL_BINOP(-, a.v - b.v, a.d[i] - b.d[i])
MD200_DUAL_BINOP(*, a.v * b.v, mul_add(a.d[i], b.v, a.v * b.d[i]))
#undef MD200_DUAL_BINOP

template <class T, int ND>
MD200_FN Dual<T, ND> mul_add(const Dual<T, ND> &a, const Dual<T, ND> &b, const Dual<T, ND> &c) {
  return a * b + c;
}

template <class T, int ND>
MD200_FN Dual<T, ND> operator/(const Dual<T, ND> &a, const Dual<T, ND> &b) {
  Dual<T, ND> r;
  const T ib = T(1) / b.v;
  r.v = a.v * ib;
#pragma unroll
  for (int i = 0; i < ND; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * ib;
  return r;
}
template <class T, int ND>
MD200_FN Dual<T, ND> operator-(const Dual<T, ND> &a) {
  Dual<T, ND> r;
  r.v = -a.v;
#pragma unroll
  for (int i = 0; i < ND; ++i) r.d[i] = -a.d[i];
  return r;
}
// Mixed with a base-type scalar
template <class T, int ND>
MD200_FN Dual<T, ND> operator*(const Dual<T, ND> &a, T s) {
  Dual<T, ND> r;
  r.v = a.v * s;
#pragma unroll
  for (int i = 0; i < ND; ++i) r.d[i] = a.d[i] * s;
  return r;
}
template <class T, int ND>
MD200_FN Dual<T, ND> operator*(T s, const Dual<T, ND> &a) { return a * s; }
template <class T, int ND>
MD200_FN Dual<T, ND> operator+(const Dual<T, ND> &a, T s) {
  Dual<T, ND> r = a;
  r.v = r.v + s;
  return r;
}
template <class T, int ND>
MD200_FN Dual<T, ND> operator+(T s, const Dual<T, ND> &a) { return a + s; }
template <class T, int ND>
MD200_FN Dual<T, ND> operator-(const Dual<T, ND> &a, T s) {
  Dual<T, ND> r = a;
  r.v = r.v - s;
  return r;
}
template <class T, int ND>
MD200_FN Dual<T, ND> operator-(T s, const Dual<T, ND> &a) {
  Dual<T, ND> r = -a;
  r.v = r.v + s;
  return r;
}
// Nested duals with a plain scalar (the innermost type)
template <class T, int ND, class S,
          typename std::enable_if<IsDual<T>::value && std::is_arithmetic<S>::value, int>::type = 0>
MD200_FN Dual<T, ND> operator*(const Dual<T, ND> &a, S s) {
  Dual<T, ND> r;
  r.v = a.v * s;
#pragma unroll
  for (int i = 0; i < ND; ++i) r.d[i] = a.d[i] * s;
  return r;
}
template <class T, int ND, class S,
          typename std::enable_if<IsDual<T>::value && std::is_arithmetic<S>::value, int>::type = 0>
MD200_FN Dual<T, ND> operator*(S s, const Dual<T, ND> &a) { return a * s; }
template <class T, int ND, class S,
          typename std::enable_if<IsDual<T>::value && std::is_arithmetic<S>::value, int>::type = 0>
MD200_FN Dual<T, ND> operator+(const Dual<T, ND> &a, S s) {
  Dual<T, ND> r = a;
  r.v = r.v + s;
  return r;
}
template <class T, int ND, class S,
          typename std::enable_if<IsDual<T>::value && std::is_arithmetic<S>::value, int>::type = 0>
MD200_FN Dual<T, ND> operator-(const Dual<T, ND> &a, S s) {
  Dual<T, ND> r = a;
  r.v = r.v - s;
  return r;
}
template <class T, int ND, class S,
          typename std::enable_if<IsDual<T>::value && std::is_arithmetic<S>::value, int>::type = 0>
MD200_FN Dual<T, ND> operator-(S s, const Dual<T, ND> &a) {
  Dual<T, ND> r = -a;
  r.v = r.v + s;
  return r;
}

// --- elementary functions --------------------------------------------------
// Double: IEEE libdevice routines.  Float: the accurate single-precision
// routines for sin/cos (argument reduction matters, phases reach ~1e3 rad) and
// the hardware approximations for exp and reciprocal square root, whose
// relative errors (~1e-7) sit far below the scan's sign-decision threshold.
#if defined(__CUDA_ARCH__)
MD200_FN double m_rsqrt(double x) { return rsqrt(x); }
MD200_FN float m_rsqrt(float x) { return rsqrtf(x); }
MD200_FN void m_sincos(double x, double *s, double *c) { sincos(x, s, c); }
// Single precision: reduce by 2 pi with a two-constant Cody-Waite split (exact
// for the |x| < 2^12 rad phases of the recurrences) and evaluate with the
// special-function unit; absolute error ~4e-7, far below the scan's
// sign-decision threshold (|g| < 2e-4 samples are re-evaluated in FP64).
MD200_FN void m_sincos(float x, float *s, float *c) {
  const float n = rintf(x * 0.15915494309189535f);
  const float r = fmaf(n, -1.7484555e-07f, fmaf(n, -6.28318548f, x));
  __sincosf(r, s, c);
}
MD200_FN double m_exp(double x) { return exp(x); }
MD200_FN float m_exp(float x) { return __expf(x); }
MD200_FN float m_expm1(float x) { return expm1f(x); }
MD200_FN double m_expm1(double x) { return expm1(x); }
#else
MD200_FN double m_rsqrt(double x) { return 1.0 / sqrt(x); }
MD200_FN float m_rsqrt(float x) { return 1.0f / sqrtf(x); }
MD200_FN void m_sincos(double x, double *s, double *c) { *s = sin(x); *c = cos(x); }
MD200_FN void m_sincos(float x, float *s, float *c) { *s = sinf(x); *c = cosf(x); }
MD200_FN double m_exp(double x) { return exp(x); }
MD200_FN float m_exp(float x) { return expf(x); }
MD200_FN float m_expm1(float x) { return expm1f(x); }
MD200_FN double m_expm1(double x) { return expm1(x); }
#endif
MD200_FN double m_sqrt(double x) { return sqrt(x); }
MD200_FN float m_sqrt(float x) { return sqrtf(x); }
MD200_FN double m_abs(double x) { return fabs(x); }
MD200_FN float m_abs(float x) { return fabsf(x); }
MD200_FN double m_max(double a, double b) { return fmax(a, b); }
MD200_FN float m_max(float a, float b) { return fmaxf(a, b); }
MD200_FN double m_log2(double x) { return log2(x); }
MD200_FN float m_log2(float x) { return log2f(x); }

template <class T, int ND>
MD200_FN Dual<T, ND> m_rsqrt(const Dual<T, ND> &x) {
  Dual<T, ND> r;
  r.v = m_rsqrt(x.v);
  const T k = T(-0.5) * r.v * r.v * r.v;
#pragma unroll
  for (int i = 0; i < ND; ++i) r.d[i] = k * x.d[i];
  return r;
}
template <class T, int ND>
MD200_FN void m_sincos(const Dual<T, ND> &x, Dual<T, ND> *s, Dual<T, ND> *c) {
  T sv, cv;
  m_sincos(x.v, &sv, &cv);
  s->v = sv;
  c->v = cv;
#pragma unroll
  for (int i = 0; i < ND; ++i) {
    s->d[i] = cv * x.d[i];
    c->d[i] = -sv * x.d[i];
  }
}
template <class T, int ND>
MD200_FN Dual<T, ND> m_exp(const Dual<T, ND> &x) {
  Dual<T, ND> r;
  r.v = m_exp(x.v);
#pragma unroll
  for (int i = 0; i < ND; ++i) r.d[i] = r.v * x.d[i];
  return r;
}
template <class T, int ND>
MD200_FN Dual<T, ND> m_sqrt(const Dual<T, ND> &x) {
  Dual<T, ND> r;
  r.v = m_sqrt(x.v);
  const T k = T(0.5) / r.v;
#pragma unroll
  for (int i = 0; i < ND; ++i) r.d[i] = k * x.d[i];
  return r;
}
template <class T, int ND>
MD200_FN Dual<T, ND> m_abs(const Dual<T, ND> &x) {
  return val(x) < 0 ? -x : x;
}

// Exact power-of-two reciprocal of the binade of x (x > 0, finite, normal):
// for x = m * 2^E with m in [1, 2) it returns 2^-E, so x * r = m lies in [1, 2)
// and the multiplication is exact.  The per-layer normalisation uses it instead
// of a division: the normalised vector has max |e_i| in [1, 2), the sign of F
// and the shape feature are unchanged.
MD200_FN double pow2_inverse(double x) {
  long long bits;
  memcpy(&bits, &x, sizeof bits);
  const long long e = (bits >> 52) & 0x7ff;
  bits = (2046LL - e) << 52;
  double r;
  memcpy(&r, &bits, sizeof r);
  return r;
}
MD200_FN float pow2_inverse(float x) {
  int bits;
  memcpy(&bits, &x, sizeof bits);
  const int e = (bits >> 23) & 0xff;
  bits = (254 - e) << 23;
  float r;
  memcpy(&r, &bits, sizeof r);
  return r;
}

// Scale the vector by the exact power of two that brings its largest component
// into [1, 2); returns the base-2 exponent removed (0 when nothing was done).
MD200_FN int binade(double x) {
  long long bits;
  memcpy(&bits, &x, sizeof bits);
  return static_cast<int>((bits >> 52) & 0x7ff) - 1023;
}
MD200_FN int binade(float x) {
  int bits;
  memcpy(&bits, &x, sizeof bits);
  return ((bits >> 23) & 0xff) - 127;
}
template <class N>
MD200_FN int scale_vector(N *e, int n, typename Base<N>::type tiny) {
  using T = typename Base<N>::type;
  T big = T(0);
#pragma unroll
  for (int i = 0; i < 5; ++i)
    if (i < n) big = m_max(big, m_abs(val(e[i])));
  if (big >= tiny && big < T(INFINITY)) {
    const T r = pow2_inverse(big);
#pragma unroll
    for (int i = 0; i < 5; ++i)
      if (i < n) e[i] = e[i] * r;
    return binade(big);
  }
  return 0;
}

// sqrt((k + kv) |k - kv|) and its reciprocal, from one reciprocal square root.
template <class N>
MD200_FN void radical(const N &k, const N &kv, N *r, N *ir) {
  using T = typename Base<N>::type;
  N d = k - kv;
  if (val(d) < T(0)) d = -d;
  const N X = (k + kv) * d;
  if (val(X) > T(0)) {
    *ir = m_rsqrt(X);
    *r = X * *ir;
  } else {
    *r = X;       // zero (with its derivative): the equal-velocity branch ignores it
    *ir = X;
  }
}

// ---------------------------------------------------------------------------
// Model view: per-layer constants prepared once per model (in shared memory).
// ---------------------------------------------------------------------------
template <class T>
struct LayerView {
  // rows of one model, each Ls long: h, 1/vp, 1/vs (0 for a fluid layer), vs^2,
  // rho, 1/rho, 1/(rho vs^2) (0 for a fluid layer)
  const T *base;
  int Ls;
  int L;      // rows including the half-space
  int water;  // 1 when row 0 is a fluid (vs = 0) layer
  MD200_FN T h(int j) const { return base[j]; }
  MD200_FN T ivp(int j) const { return base[Ls + j]; }
  MD200_FN T ivs(int j) const { return base[2 * Ls + j]; }
  MD200_FN T vs2(int j) const { return base[3 * Ls + j]; }
  MD200_FN T rho(int j) const { return base[4 * Ls + j]; }
  MD200_FN T irho(int j) const { return base[5 * Ls + j]; }
  MD200_FN T imu(int j) const { return base[6 * Ls + j]; }
};

// The 15 distinct entries of one layer's Dunkin compound matrix; the 5x5
// matrix acting on the column vector e is
//   [A E tJ F O; D B tH N F; I G K H J; C M tG B E; L C tI D A],  t = -2 k^2
// (the column of e[2] carries t outside the K entry).
template <class N>
struct RayleighEntries {
  N A, B, C, D, E, F, G, H, I, J, K, Lm, M, Nn, O;
};

// One wave (P or S) of a layer at wavenumber k against the layer's wavenumber kv:
// cs = cos(r h), sr = sin(r h) / r, rs = -r sin(r h) for a propagating wave
// (k < kv); for an evanescent one the hyperbolic forms scaled by
// scale = exp(-r h): cs = (1 + e^2) / 2, sr = (1 - e^2) / (2 r), rs = r (1 - e^2) / 2,
// and the return value is r h (value part), the exponent factored out; at
// k = kv the limits 1, h, 0.  r = sqrt((k + kv)|k - kv|).  scale is 1 unless
// evanescent.
//
// Near k = kv derivative-carrying numbers take the power series in
// y = (k^2 - kv^2) h^2 instead, unscaled and without the square root:
//   cs = C(y), sr = h S(y), rs = (k^2 - kv^2) h S(y),
//   C(y) = sum y^n / (2n)!, S(y) = sum y^n / (2n+1)!
// (cos and sin for y < 0, cosh and sinh for y > 0).  The direct form takes
// sin(r h) / r through r = sqrt(|k^2 - kv^2|), and the two terms of its
// derivative cancel to a relative error of about eps / (r h)^2: for a root 1e-8
// below a layer's velocity that moved group velocities by 1e-6.  Plain numbers
// (values) keep the direct forms, so root sets are unaffected.  Every dual type
// takes the same branch (the adjoint Jacobians recompute blocks in several
// number types, which must agree on the scaling).  The band is narrow because
// thin layers at long periods have small y at every velocity, and the series
// costs more than the direct form in the adjoint's nested duals: at
// |y| = WAVE_SERIES_Y the direct form's cancellation is eps / |y| ~ 2e-12, and
// truncation after y^3 leaves < 3e-21 relative error inside the band.
constexpr double WAVE_SERIES_Y = 1e-4;

template <class N, class T>
MD200_FN bool wave_series(const N &k, const N &kv, T h, N *cs, N *sr, N *rs) {
  using BT = typename Base<N>::type;
  const BT kk = val(k), kvv = val(kv), hh = val(h);
  const BT yv = (((kk + kvv) * (kk - kvv)) * hh) * hh;  // the value part of y, decided on first
  if (!(yv < BT(WAVE_SERIES_Y) && yv > -BT(WAVE_SERIES_Y))) return false;
  const N D = (k + kv) * (k - kv);
  const N y = (D * h) * h;
  N C = y * BT(1. / 720.) + BT(1. / 24.);  // 1/6!, 1/4!
  C = C * y + BT(0.5);
  *cs = C * y + BT(1);
  N S = y * BT(1. / 5040.) + BT(1. / 120.);  // 1/7!, 1/5!
  S = S * y + BT(1. / 6.);
  S = S * y + BT(1);
  *sr = S * h;
  *rs = (D * S) * h;
  return true;
}

template <class N, class T>
MD200_FN typename Base<N>::type wave_block(const N &k, const N &kv, T h, N *cs, N *sr, N *rs, N *scale) {
  using BT = typename Base<N>::type;
  if constexpr (IsDual<N>::value) {
    if (wave_series<N, T>(k, kv, h, cs, sr, rs)) {
      *scale = lift_one<N>();
      return BT(0);
    }
  }
  N r, ir;
  radical(k, kv, &r, &ir);
  *scale = lift_one<N>();
  if (val(k) < val(kv)) {
    N sn;
    m_sincos(r * h, &sn, cs);
    *sr = sn * ir;
    *rs = -(r * sn);
    return BT(0);
  }
  if (val(k) == val(kv)) {
    *cs = lift_one<N>();
    *sr = lift_one<N>() * h;
    *rs = lift_zero<N>();
    return BT(0);
  }
  const N e = m_exp(-(r * h));
  const N fac = e * e;
  *cs = (fac + BT(1)) * BT(0.5);
  const N sh = (BT(1) - fac) * BT(0.5);
  *sr = sh * ir;
  *rs = r * sh;
  *scale = e;
  return val(r) * val(h);
}

// The 15 entries from the wave blocks (cosp, wv = sin_p/r_p, xv = -r_p sin_p;
// cosq, yv, zv likewise for S; a0 the product of the evanescent scales),
// gam = 2 k^2 vs^2 / w^2, gammk = gam / k^2, and the density.
template <class N, class T>
MD200_FN void rayleigh_poly(RayleighEntries<N> &X, const N &cosp, const N &wv, const N &xv, const N &cosq,
                            const N &yv, const N &zv, const N &a0, const N &gam, const N &gammk, const N &k2,
                            T rho, T irho) {
  using BT = typename Base<N>::type;
  const N cpcq = cosp * cosq, cpy = cosp * yv, cpz = cosp * zv;
  const N cqw = cosq * wv, cqx = cosq * xv;
  const N xy = xv * yv, xz = xv * zv, wy = wv * yv, wz = wv * zv;

  const N gm1 = gam - BT(1);
  const N twgm1 = gam + gm1;
  const N gmgmk = gam * gammk;
  const N gmgm1 = gam * gm1;
  const N gm1sq = gm1 * gm1;
  const N a0pq = a0 - cpcq;
  const T rho2 = rho * rho, irho2 = irho * irho;

  X.A = cpcq - (gmgm1 * a0pq) * BT(2) - gmgmk * xz - k2 * gm1sq * wy;
  X.D = (k2 * cpy - cqx) * irho;
  X.I = -(twgm1 * a0pq + gammk * xz + k2 * gm1 * wy) * irho;
  X.C = (cpz - k2 * cqw) * irho;
  X.Lm = -((k2 * a0pq) * BT(2) + xz + k2 * k2 * wy) * irho2;
  X.E = (gmgmk * cpz - gm1sq * cqw) * rho;
  X.G = gammk * cpz - gm1 * cqw;
  X.M = -wz;
  X.Nn = -xy;
  X.F = (gm1sq * cpy - gmgmk * cqx) * rho;
  X.H = gm1 * cpy - gammk * cqx;
  X.O = -((gmgmk * gm1sq * a0pq) * BT(2) + gmgmk * gmgmk * xz + gm1sq * gm1sq * wy) * rho2;
  X.J = -(gammk * gm1 * twgm1 * a0pq + gam * gammk * gammk * xz + gm1 * gm1sq * wy) * rho;
  X.K = a0 + (cpcq - X.A) * BT(2);
  X.B = cpcq;
}

// Entries of layer (h, 1/vp, vs^2, 1/vs, rho, 1/rho) at wavenumber k (k2 = k^2),
// frequency w (iw2 = 1/w^2).  Returns the exponent P + Q (value part) that the
// scaled hyperbolic functions of the evanescent branches factor out: the
// unscaled matrix is the returned one times exp(P + Q).  The layer constants may
// be plain numbers or numbers of type N (parameter derivatives).
template <class N, class T>
MD200_FN typename Base<N>::type rayleigh_entries(RayleighEntries<N> &X, const N &k, const N &k2,
                                                 const N &w, const N &iw2, T h, T ivp, T vs2, T ivs,
                                                 T rho, T irho) {
  using BT = typename Base<N>::type;
  const N ka = w * ivp, kb = w * ivs;
  const N gammk = (iw2 * vs2) * BT(2);
  const N gam = gammk * k2;
  N cosp, wv, xv, ep, cosq, yv, zv, eq;
  const BT expo = wave_block<N, T>(k, ka, h, &cosp, &wv, &xv, &ep) + wave_block<N, T>(k, kb, h, &cosq, &yv, &zv, &eq);
  rayleigh_poly<N, T>(X, cosp, wv, xv, cosq, yv, zv, ep * eq, gam, gammk, k2, rho, irho);
  return expo;
}

// e <- M e for the matrix of RayleighEntries.
template <class N>
MD200_FN void rayleigh_apply(const RayleighEntries<N> &X, const N &k2, N e[5]) {
  using BT = typename Base<N>::type;
  const N e0 = e[0], e1 = e[1], e4 = e[4], e3 = e[3];
  const N e2t = e[2] * (k2 * BT(-2));
  e[0] = X.A * e0 + X.E * e1 + X.J * e2t + X.F * e3 + X.O * e4;
  e[1] = X.D * e0 + X.B * e1 + X.H * e2t + X.Nn * e3 + X.F * e4;
  e[2] = X.I * e0 + X.G * e1 + X.K * e[2] + X.H * e3 + X.J * e4;
  e[3] = X.C * e0 + X.M * e1 + X.G * e2t + X.B * e3 + X.E * e4;
  e[4] = X.Lm * e0 + X.C * e1 + X.I * e2t + X.D * e3 + X.A * e4;
}

// One upward Dunkin step through a layer: e <- e * Ca(m); returns P + Q as
// rayleigh_entries does.
template <class N, class T>
MD200_FN typename Base<N>::type rayleigh_layer(N e[5], const N &k, const N &k2, const N &w,
                                               const N &iw2, T h, T ivp, T vs2, T ivs, T rho,
                                               T irho) {
  RayleighEntries<N> X;
  const auto expo = rayleigh_entries<N, T>(X, k, k2, w, iw2, h, ivp, vs2, ivs, rho, irho);
  rayleigh_apply<N>(X, k2, e);
  return expo;
}

// Branch-free single-precision form of rayleigh_layer: both the trigonometric
// (propagating) and the scaled hyperbolic (evanescent) forms of each wave are
// evaluated with the special-function unit and selected, so the lanes of a warp
// at different velocities do not diverge.  Same matrix, same return value.
MD200_FN float rayleigh_layer_f32(float e[5], float k, float k2, float w, float iw2, float h, float ivp,
                                  float vs2, float ivs, float rho, float irho) {
  const float ka = w * ivp, kb = w * ivs;
  const float gammk = (iw2 * vs2) * 2.f;
  const float gam = gammk * k2;
  // radicals and reciprocals (zero where k equals the wavenumber exactly)
  const float Xa = (k + ka) * fabsf(k - ka), Xb = (k + kb) * fabsf(k - kb);
  const float ira = Xa > 0.f ? rsqrtf(Xa) : 0.f, irb = Xb > 0.f ? rsqrtf(Xb) : 0.f;
  const float ra = Xa * ira, rb = Xb * irb;
  const float p = ra * h, q = rb * h;
  const bool pp = k < ka, pq = k < kb;  // propagating P / S
  float sp, cp, sq, cq;
  m_sincos(p, &sp, &cp);
  m_sincos(q, &sq, &cq);
  const float ep = m_exp(-p), eq = m_exp(-q);
  const float fp = ep * ep, fq = eq * eq;
  const float cosp = pp ? cp : .5f * (1.f + fp), sinp = pp ? sp : .5f * (1.f - fp);
  const float cosq = pq ? cq : .5f * (1.f + fq), sinq = pq ? sq : .5f * (1.f - fq);
  // sin(r h)/r -> h as r -> 0
  const float wv = Xa > 0.f ? sinp * ira : h, xv = pp ? -(ra * sinp) : ra * sinp;
  const float yv = Xb > 0.f ? sinq * irb : h, zv = pq ? -(rb * sinq) : rb * sinq;
  const float a0 = (pp ? 1.f : ep) * (pq ? 1.f : eq);
  const float expo = (pp ? 0.f : p) + (pq ? 0.f : q);
  const float cpcq = cosp * cosq, cpy = cosp * yv, cpz = cosp * zv;
  const float cqw = cosq * wv, cqx = cosq * xv;
  const float xy = xv * yv, xz = xv * zv, wy = wv * yv, wz = wv * zv;
  const float gm1 = gam - 1.f, twgm1 = gam + gm1, gmgmk = gam * gammk, gmgm1 = gam * gm1, gm1sq = gm1 * gm1;
  const float a0pq = a0 - cpcq;
  const float rho2 = rho * rho, irho2 = irho * irho;
  const float A = cpcq - (gmgm1 * a0pq) * 2.f - gmgmk * xz - k2 * gm1sq * wy;
  const float D = (k2 * cpy - cqx) * irho;
  const float I = -(twgm1 * a0pq + gammk * xz + k2 * gm1 * wy) * irho;
  const float C = (cpz - k2 * cqw) * irho;
  const float Lm = -((k2 * a0pq) * 2.f + xz + k2 * k2 * wy) * irho2;
  const float E = (gmgmk * cpz - gm1sq * cqw) * rho;
  const float G = gammk * cpz - gm1 * cqw;
  const float M = -wz, Nn = -xy;
  const float F = (gm1sq * cpy - gmgmk * cqx) * rho;
  const float H = gm1 * cpy - gammk * cqx;
  const float O = -((gmgmk * gm1sq * a0pq) * 2.f + gmgmk * gmgmk * xz + gm1sq * gm1sq * wy) * rho2;
  const float J = -(gammk * gm1 * twgm1 * a0pq + gam * gammk * gammk * xz + gm1 * gm1sq * wy) * rho;
  const float K = a0 + (cpcq - A) * 2.f;
  const float B = cpcq;
  const float e0 = e[0], e1 = e[1], e3 = e[3], e4 = e[4];
  const float e2t = e[2] * (k2 * -2.f);
  e[0] = A * e0 + E * e1 + J * e2t + F * e3 + O * e4;
  e[1] = D * e0 + B * e1 + H * e2t + Nn * e3 + F * e4;
  e[2] = I * e0 + G * e1 + K * e[2] + H * e3 + J * e4;
  e[3] = C * e0 + M * e1 + G * e2t + B * e3 + E * e4;
  e[4] = Lm * e0 + C * e1 + I * e2t + D * e3 + A * e4;
  return expo;
}

// The same layer step for a layer in which both waves are deeply evanescent
// (c well below vs), in single precision.  With u = (c/vp)^2, v = (c/vs)^2, p = sqrt(1-u),
// s = sqrt(1-v), R = p s and g = 2/v (the standard form's gamma), the standard
// entries are sums of terms growing like g^4 that cancel down to O(g^2); here each
// entry is written through the exactly-computed differences 1 - R (loss),
// v - u (contrast) and the exponential differences of the two phases, so no
// cancellation occurs (the factorisation of cpp/common/dunkin.hpp:286-331).
MD200_FN float rayleigh_layer_evanescent(float e[5], float k, float k2, float c, float h, float ivp,
                                         float ivs, float rho, float irho) {
  const float cp = c * ivp, cs = c * ivs, u = cp * cp, v = cs * cs;
  const float p = sqrtf(1.f - u), s = sqrtf(1.f - v), R = p * s;
  const float loss = (u + (1.f - u) * v) / (1.f + R);
  const float g = 2.f / v, contrast = v - u;
  const float kh = k * h, q = kh * s;
  float sp = .5f, sq = .5f, a0 = 0.f, delta = 0.f, gap = 0.f;
  if (q < 16.f) {
    const float pq = kh * contrast / (p + s);  // P - Q, the phase difference
    const float eq = m_exp(-q), diff = -eq * m_expm1(-pq);
    sp = -.5f * m_expm1(-2.f * (q + pq));
    sq = -.5f * m_expm1(-2.f * q);
    a0 = eq * (eq - diff);
    delta = -.5f * diff * (2.f * eq - diff);  // cos_p sin_q - cos_q sin_p (scaled)
    gap = .5f * diff * diff;                  // cos_p cos_q - a0 - sin_p sin_q (scaled)
  }
  const float gm1 = g - 1.f, twgm1 = g + gm1;
  const float gl = g * loss;
  const float d1 = 1.f - gl, d2 = g * (2.f - gl) - 1.f;
  const float ps = sp * sq, psr = ps / R, y = (1.f - sq) * sp, x = (1.f - sp) * sq;
  const float q1 = 2.f * g * gm1 * gap, q2 = psr * d1 * d1;
  const float kp = k / p, ks = k / s, ip = 1.f / (k * p), is = 1.f / (k * s);
  const float rho2 = rho * rho, irho2 = irho * irho, ik2 = 1.f / k2;
  const float B = (1.f - sp) * (1.f - sq), A = B + q1 - q2;
  const float D = ks * (delta + loss * y) * irho, C = kp * (delta - loss * x) * irho;
  const float G = (g * R * delta + d1 * y) * ip, H = (gm1 * delta - d1 * y) * is;
  const float E = (g * g * R * delta + d2 * y) * ip * rho, F = (gm1 * gm1 * delta - d2 * y) * is * rho;
  const float I = (twgm1 * gap + psr * loss * d1) * irho;
  const float Lm = k2 * (2.f * gap - psr * loss * loss) * irho2;
  const float J = (g * gm1 * twgm1 * gap - psr * d1 * d2) * rho * ik2;
  const float O = (g * gm1 * q1 - psr * d2 * d2) * rho2 * ik2;
  const float K = a0 + 2.f * (q2 - q1), M = -ps * (s / p), Nn = -ps * (p / s);
  const float e0 = e[0], e1 = e[1], e3 = e[3], e4 = e[4];
  const float e2t = e[2] * (-2.f * k2);
  e[0] = A * e0 + E * e1 + J * e2t + F * e3 + O * e4;
  e[1] = D * e0 + B * e1 + H * e2t + Nn * e3 + F * e4;
  e[2] = I * e0 + G * e1 + K * e[2] + H * e3 + J * e4;
  e[3] = C * e0 + M * e1 + G * e2t + B * e3 + E * e4;
  e[4] = Lm * e0 + C * e1 + I * e2t + D * e3 + A * e4;
  return kh * (p + s);  // P + Q
}

// Single-precision layers switch to the factored step where c < vs / RATIO.
// Measured against the FP64 oracle on crustal and low-velocity-layer models,
// the standard step keeps every FP32 sign down to c = vs/16 and loses signs
// below about vs/64; the factored step costs ~3x a standard one, so it is used
// only where needed.
#ifndef MD200_EVANESCENT_RATIO
#define MD200_EVANESCENT_RATIO 16.f
#endif

// Fluid top layer (thickness h0, 1/vp ivp0): cos and sin/r of its P phase, the
// factors that turn the solid-stack vector into the fluid-top secular value
// cp e[0] - wv rho0 e[1].
template <class N, class T>
MD200_FN void water_top(const N &k, const N &w, T h0, T ivp0, N *cp, N *wv) {
  using B = typename Base<N>::type;
  const N ka = w * ivp0;
  if constexpr (IsDual<N>::value) {
    N rs;
    if (wave_series<N, T>(k, ka, h0, cp, wv, &rs)) return;
  }
  N rf, irf;
  radical(k, ka, &rf, &irf);
  if (val(k) < val(ka)) {
    N sn;
    m_sincos(rf * h0, &sn, cp);
    *wv = sn * irf;
  } else if (val(k) == val(ka)) {
    *cp = lift_one<N>();
    *wv = lift_one<N>() * h0;
  } else {
    const N ez = m_exp(-(rf * h0));
    const N z = ez * ez;
    *cp = (z + B(1)) * B(0.5);
    *wv = ((B(1) - z) * B(0.5)) * irf;
  }
}

// Half-space start vector of the upward sweep (half-space 1/vp, 1/vs, vs^2, rho).
template <class N, class T>
MD200_FN void rayleigh_start(N e[5], const N &k, const N &k2, const N &w, const N &iw2, T ivp, T ivs,
                             T vs2, T rh) {
  const N ka = w * ivp, kb = w * ivs;
  N ra, ira, rb, irb;
  radical(k, ka, &ra, &ira);
  radical(k, kb, &rb, &irb);
  const N gammk = (iw2 * vs2) * T(2);
  const N gam = gammk * k2;
  const N gm1 = gam - T(1);
  const N rarb = ra * rb;
  e[0] = (gm1 * gm1 - gam * gammk * rarb) * (rh * rh);
  e[1] = -(ra * rh);
  e[2] = (gm1 - gammk * rarb) * rh;
  e[3] = rb * rh;
  e[4] = k2 - rarb;
}

// ---------------------------------------------------------------------------
// Explicitly rounded single precision for the scan's Rayleigh evaluations.
// Every addition, multiplication and fused multiply-add of the recurrence is
// one PTX instruction with round-to-nearest and flush-to-zero, so no compiler
// contraction chooses a rounding.  The arithmetic is written once over a lane
// type: R1 carries one sample per thread, R2 two samples of the same trace per
// thread in sm_100's paired single-precision instructions (add/mul/fma .f32x2,
// one issue slot for both samples).  Per-lane work -- special functions,
// comparisons, selections, the power-of-two normalisation -- runs on each half
// with the same scalar code.  Each half of an R2 result is therefore bit for bit
// the R1 result of that sample: the split scan's paired evaluations and the
// fused scan's single ones return the same values.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float x_mul(float a, float b) {
  float r;
  asm("mul.rn.ftz.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ float x_add(float a, float b) {
  float r;
  asm("add.rn.ftz.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ float x_fma(float a, float b, float c) {
  float r;
  asm("fma.rn.ftz.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}

struct R1 {
  using V = float;
  static constexpr int NL = 1;
  using M = bool;
  static __device__ __forceinline__ V mul(V a, V b) { return x_mul(a, b); }
  static __device__ __forceinline__ V add(V a, V b) { return x_add(a, b); }
  static __device__ __forceinline__ V fma(V a, V b, V c) { return x_fma(a, b, c); }
  static __device__ __forceinline__ V splat(float a) { return a; }
  static __device__ __forceinline__ V neg(V a) { return -a; }
  static __device__ __forceinline__ V abs(V a) { return fabsf(a); }
  static __device__ __forceinline__ M lt(V a, float b) { return a < b; }
  static __device__ __forceinline__ M gt0(V a) { return a > 0.f; }
  static __device__ __forceinline__ V sel(M m, V a, V b) { return m ? a : b; }
  static __device__ __forceinline__ V rsqrt0(V a) { return a > 0.f ? rsqrtf(a) : 0.f; }
  static __device__ __forceinline__ V expneg(V a) { return __expf(-a); }
  static __device__ __forceinline__ V rint(V a) { return rintf(a); }
  static __device__ __forceinline__ void sincos(V r, V *s, V *c) { __sincosf(r, s, c); }
};

struct R2 {
  using V = float2;
  static constexpr int NL = 2;
  struct M {
    bool x, y;
  };
  static __device__ __forceinline__ unsigned long long pk(V a) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
    return r;
  }
  static __device__ __forceinline__ V upk(unsigned long long r) {
    V a;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(r));
    return a;
  }
  static __device__ __forceinline__ V mul(V a, V b) {
    unsigned long long r;
    asm("mul.rn.ftz.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pk(a)), "l"(pk(b)));
    return upk(r);
  }
  static __device__ __forceinline__ V add(V a, V b) {
    unsigned long long r;
    asm("add.rn.ftz.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pk(a)), "l"(pk(b)));
    return upk(r);
  }
  static __device__ __forceinline__ V fma(V a, V b, V c) {
    unsigned long long r;
    asm("fma.rn.ftz.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(pk(a)), "l"(pk(b)), "l"(pk(c)));
    return upk(r);
  }
  static __device__ __forceinline__ V splat(float a) { return make_float2(a, a); }
  static __device__ __forceinline__ V neg(V a) { return make_float2(-a.x, -a.y); }
  static __device__ __forceinline__ V abs(V a) { return make_float2(fabsf(a.x), fabsf(a.y)); }
  static __device__ __forceinline__ M lt(V a, float b) { return {a.x < b, a.y < b}; }
  static __device__ __forceinline__ M gt0(V a) { return {a.x > 0.f, a.y > 0.f}; }
  static __device__ __forceinline__ V sel(M m, V a, V b) { return make_float2(m.x ? a.x : b.x, m.y ? a.y : b.y); }
  static __device__ __forceinline__ V rsqrt0(V a) { return make_float2(R1::rsqrt0(a.x), R1::rsqrt0(a.y)); }
  static __device__ __forceinline__ V expneg(V a) { return make_float2(__expf(-a.x), __expf(-a.y)); }
  static __device__ __forceinline__ V rint(V a) { return make_float2(rintf(a.x), rintf(a.y)); }
  static __device__ __forceinline__ void sincos(V r, V *s, V *c) {
    __sincosf(r.x, &s->x, &c->x);
    __sincosf(r.y, &s->y, &c->y);
  }
};

// sin and cos of a phase: reduction by 2 pi with a two-constant Cody-Waite split
// (exact for the |x| < 2^12 rad phases of the recurrences), then the
// special-function unit (absolute error ~4e-7, far below the scan's
// sign-decision threshold).
template <class P>
__device__ __forceinline__ void sincos32(typename P::V x, typename P::V *s, typename P::V *c) {
  const typename P::V n = P::rint(P::mul(x, P::splat(0.15915494309189535f)));
  const typename P::V r = P::fma(n, P::splat(-1.7484555e-07f), P::fma(n, P::splat(-6.28318548f), x));
  P::sincos(r, s, c);
}

// e <- M e for the 15 entries (t = -2 k^2 carried by the e[2] column).
template <class P>
__device__ __forceinline__ void apply32(typename P::V e[5], typename P::V k2, typename P::V A, typename P::V B,
                                        typename P::V C, typename P::V D, typename P::V E, typename P::V F,
                                        typename P::V G, typename P::V H, typename P::V I, typename P::V J,
                                        typename P::V K, typename P::V Lm, typename P::V M, typename P::V Nn,
                                        typename P::V O) {
  const typename P::V e0 = e[0], e1 = e[1], e2 = e[2], e3 = e[3], e4 = e[4];
  const typename P::V e2t = P::mul(e2, P::mul(k2, P::splat(-2.f)));
  e[0] = P::fma(O, e4, P::fma(F, e3, P::fma(J, e2t, P::fma(E, e1, P::mul(A, e0)))));
  e[1] = P::fma(F, e4, P::fma(Nn, e3, P::fma(H, e2t, P::fma(B, e1, P::mul(D, e0)))));
  e[2] = P::fma(J, e4, P::fma(H, e3, P::fma(K, e2, P::fma(G, e1, P::mul(I, e0)))));
  e[3] = P::fma(E, e4, P::fma(B, e3, P::fma(G, e2t, P::fma(M, e1, P::mul(C, e0)))));
  e[4] = P::fma(A, e4, P::fma(D, e3, P::fma(I, e2t, P::fma(C, e1, P::mul(Lm, e0)))));
}

// One standard Dunkin layer step (both waves trigonometric or scaled
// hyperbolic, selected per lane), the algebra of rayleigh_layer_f32.  ka, kb,
// gammk and the density powers are the layer's per-trace constants.  Returns
// the exponent P + Q factored out of the evanescent waves.
template <class P>
__device__ __forceinline__ typename P::V step32(typename P::V e[5], typename P::V k, typename P::V k2, float ka,
                                                float kb, float gammk, float h, float rho, float irho, float rho2,
                                                float irho2) {
  using V = typename P::V;
  const V one = P::splat(1.f), zero = P::splat(0.f), half = P::splat(.5f), mhalf = P::splat(-.5f);
  const V gam = P::mul(P::splat(gammk), k2);
  const V Xa = P::mul(P::add(k, P::splat(ka)), P::abs(P::add(k, P::splat(-ka))));
  const V Xb = P::mul(P::add(k, P::splat(kb)), P::abs(P::add(k, P::splat(-kb))));
  const V ira = P::rsqrt0(Xa), irb = P::rsqrt0(Xb);
  const V ra = P::mul(Xa, ira), rb = P::mul(Xb, irb);
  const V p = P::mul(ra, P::splat(h)), q = P::mul(rb, P::splat(h));
  V sp, cp, sq, cq;
  sincos32<P>(p, &sp, &cp);
  sincos32<P>(q, &sq, &cq);
  const V ep = P::expneg(p), eq = P::expneg(q);
  const V fp = P::mul(ep, ep), fq = P::mul(eq, eq);
  const typename P::M pp = P::lt(k, ka), pq = P::lt(k, kb);  // propagating P / S
  const V cosp = P::sel(pp, cp, P::fma(fp, half, half)), sinp = P::sel(pp, sp, P::fma(fp, mhalf, half));
  const V cosq = P::sel(pq, cq, P::fma(fq, half, half)), sinq = P::sel(pq, sq, P::fma(fq, mhalf, half));
  // sin(r h)/r -> h as r -> 0
  const V wv = P::sel(P::gt0(Xa), P::mul(sinp, ira), P::splat(h));
  const V yv = P::sel(P::gt0(Xb), P::mul(sinq, irb), P::splat(h));
  const V tp = P::mul(ra, sinp), tq = P::mul(rb, sinq);
  const V xv = P::sel(pp, P::neg(tp), tp), zv = P::sel(pq, P::neg(tq), tq);
  const V a0 = P::mul(P::sel(pp, one, ep), P::sel(pq, one, eq));
  const V expo = P::add(P::sel(pp, zero, p), P::sel(pq, zero, q));
  const V cpcq = P::mul(cosp, cosq), cpy = P::mul(cosp, yv), cpz = P::mul(cosp, zv);
  const V cqw = P::mul(cosq, wv), cqx = P::mul(cosq, xv);
  const V xy = P::mul(xv, yv), xz = P::mul(xv, zv), wy = P::mul(wv, yv), wz = P::mul(wv, zv);
  const V gmk = P::splat(gammk);
  const V gm1 = P::add(gam, P::splat(-1.f)), twgm1 = P::add(gam, gm1);
  const V gmgmk = P::mul(gam, gmk), gmgm1 = P::mul(gam, gm1), gm1sq = P::mul(gm1, gm1);
  const V a0pq = P::add(a0, P::neg(cpcq));
  const V k2gm1 = P::mul(k2, gm1), k2gm1sq = P::mul(k2, gm1sq);
  V A = P::fma(P::mul(gmgm1, P::splat(-2.f)), a0pq, cpcq);
  A = P::fma(P::neg(gmgmk), xz, A);
  A = P::fma(P::neg(k2gm1sq), wy, A);
  const V D = P::mul(P::fma(k2, cpy, P::neg(cqx)), P::splat(irho));
  const V I = P::mul(P::fma(k2gm1, wy, P::fma(twgm1, a0pq, P::mul(gmk, xz))), P::splat(-irho));
  const V C = P::mul(P::fma(P::neg(k2), cqw, cpz), P::splat(irho));
  const V Lm = P::mul(P::fma(P::mul(k2, k2), wy, P::fma(P::mul(k2, P::splat(2.f)), a0pq, xz)), P::splat(-irho2));
  const V E = P::mul(P::fma(gmgmk, cpz, P::neg(P::mul(gm1sq, cqw))), P::splat(rho));
  const V G = P::fma(gmk, cpz, P::neg(P::mul(gm1, cqw)));
  const V F = P::mul(P::fma(gm1sq, cpy, P::neg(P::mul(gmgmk, cqx))), P::splat(rho));
  const V H = P::fma(gm1, cpy, P::neg(P::mul(gmk, cqx)));
  const V gg = P::mul(gmgmk, gm1sq);
  const V O = P::mul(P::fma(P::mul(gm1sq, gm1sq), wy, P::fma(P::mul(gg, P::splat(2.f)), a0pq,
                                                             P::mul(P::mul(gmgmk, gmgmk), xz))),
                     P::splat(-rho2));
  const V J = P::mul(P::fma(P::mul(gm1, gm1sq), wy, P::fma(P::mul(P::mul(gmk, gm1), twgm1), a0pq,
                                                           P::mul(P::mul(gmgmk, gmk), xz))),
                     P::splat(-rho));
  const V K = P::fma(P::splat(2.f), P::add(cpcq, P::neg(A)), a0);
  apply32<P>(e, k2, A, cpcq, C, D, E, F, G, H, I, J, K, Lm, P::neg(wz), P::neg(xy), O);
  return expo;
}

// The factored step of rayleigh_layer_evanescent (both waves deeply evanescent,
// c < vs / MD200_EVANESCENT_RATIO) for one sample, explicitly rounded.
__device__ __forceinline__ float evanescent32(float e[5], float k, float k2, float c, float h, float ivp, float ivs,
                                              float rho, float irho, float rho2, float irho2) {
  const float cp = x_mul(c, ivp), cs = x_mul(c, ivs), u = x_mul(cp, cp), v = x_mul(cs, cs);
  const float p = sqrtf(x_add(1.f, -u)), s = sqrtf(x_add(1.f, -v)), R = x_mul(p, s);
  const float loss = x_fma(x_add(1.f, -u), v, u) / x_add(1.f, R);
  const float g = 2.f / v, contrast = x_add(v, -u);
  const float kh = x_mul(k, h), q = x_mul(kh, s);
  float sp = .5f, sq = .5f, a0 = 0.f, delta = 0.f, gap = 0.f;
  if (q < 16.f) {
    const float pq = x_mul(kh, contrast) / x_add(p, s);  // P - Q, the phase difference
    const float eq = __expf(-q), diff = x_mul(-eq, expm1f(-pq));
    sp = x_mul(-.5f, expm1f(x_mul(-2.f, x_add(q, pq))));
    sq = x_mul(-.5f, expm1f(x_mul(-2.f, q)));
    a0 = x_mul(eq, x_add(eq, -diff));
    delta = x_mul(x_mul(-.5f, diff), x_fma(2.f, eq, -diff));  // cos_p sin_q - cos_q sin_p (scaled)
    gap = x_mul(x_mul(.5f, diff), diff);                       // cos_p cos_q - a0 - sin_p sin_q (scaled)
  }
  const float gm1 = x_add(g, -1.f), twgm1 = x_add(g, gm1);
  const float gl = x_mul(g, loss);
  const float d1 = x_add(1.f, -gl), d2 = x_fma(g, x_add(2.f, -gl), -1.f);
  const float ps = x_mul(sp, sq), psr = ps / R;
  const float y = x_mul(x_add(1.f, -sq), sp), x = x_mul(x_add(1.f, -sp), sq);
  const float q1 = x_mul(x_mul(x_mul(2.f, g), gm1), gap), q2 = x_mul(x_mul(psr, d1), d1);
  const float kp = k / p, ks = k / s, ip = 1.f / x_mul(k, p), is = 1.f / x_mul(k, s), ik2 = 1.f / k2;
  const float B = x_mul(x_add(1.f, -sp), x_add(1.f, -sq)), A = x_add(x_add(B, q1), -q2);
  const float D = x_mul(x_mul(ks, x_fma(loss, y, delta)), irho);
  const float C = x_mul(x_mul(kp, x_fma(-loss, x, delta)), irho);
  const float G = x_mul(x_fma(x_mul(g, R), delta, x_mul(d1, y)), ip);
  const float H = x_mul(x_fma(gm1, delta, -x_mul(d1, y)), is);
  const float E = x_mul(x_mul(x_fma(x_mul(x_mul(g, g), R), delta, x_mul(d2, y)), ip), rho);
  const float F = x_mul(x_mul(x_fma(x_mul(gm1, gm1), delta, -x_mul(d2, y)), is), rho);
  const float I = x_mul(x_fma(twgm1, gap, x_mul(x_mul(psr, loss), d1)), irho);
  const float Lm = x_mul(x_mul(k2, x_fma(2.f, gap, -x_mul(x_mul(psr, loss), loss))), irho2);
  const float J = x_mul(x_mul(x_fma(x_mul(x_mul(g, gm1), twgm1), gap, -x_mul(x_mul(psr, d1), d2)), rho), ik2);
  const float O = x_mul(x_mul(x_fma(x_mul(g, gm1), q1, -x_mul(x_mul(psr, d2), d2)), rho2), ik2);
  const float K = x_fma(2.f, x_add(q2, -q1), a0);
  const float M = x_mul(-ps, s / p), Nn = x_mul(-ps, p / s);
  apply32<R1>(e, k2, A, B, C, D, E, F, G, H, I, J, K, Lm, M, Nn, O);
  return x_mul(kh, x_add(p, s));  // P + Q
}

// Per-lane access to a lane type's values.
__device__ __forceinline__ float &lane_of(float &v, int) { return v; }
__device__ __forceinline__ float &lane_of(float2 &v, int i) { return i ? v.y : v.x; }
__device__ __forceinline__ float lane_of(const float &v, int) { return v; }
__device__ __forceinline__ float lane_of(const float2 &v, int i) { return i ? v.y : v.x; }

// Half-space start vector (the standard form, then per lane the factored form
// well below the shear velocity).
template <class P>
__device__ __forceinline__ void start32(typename P::V e[5], typename P::V k, typename P::V k2, typename P::V c,
                                        float w, float iw2, float ivp, float ivs, float vs2, float rh) {
  using V = typename P::V;
  const float ka = x_mul(w, ivp), kb = x_mul(w, ivs), gammk = x_mul(x_mul(iw2, vs2), 2.f), rh2 = x_mul(rh, rh);
  const V Xa = P::mul(P::add(k, P::splat(ka)), P::abs(P::add(k, P::splat(-ka))));
  const V Xb = P::mul(P::add(k, P::splat(kb)), P::abs(P::add(k, P::splat(-kb))));
  const V ra = P::mul(Xa, P::rsqrt0(Xa)), rb = P::mul(Xb, P::rsqrt0(Xb));
  const V gam = P::mul(P::splat(gammk), k2), gm1 = P::add(gam, P::splat(-1.f)), rarb = P::mul(ra, rb);
  e[0] = P::mul(P::fma(gm1, gm1, P::neg(P::mul(P::mul(gam, P::splat(gammk)), rarb))), P::splat(rh2));
  e[1] = P::mul(ra, P::splat(-rh));
  e[2] = P::mul(P::fma(P::splat(-gammk), rarb, gm1), P::splat(rh));
  e[3] = P::mul(rb, P::splat(rh));
  e[4] = P::add(k2, P::neg(rarb));
#pragma unroll
  for (int i = 0; i < P::NL; ++i) {
    const float cc = lane_of(c, i), kk = lane_of(k, i);
    if (x_mul(x_mul(MD200_EVANESCENT_RATIO, cc), ivs) < 1.f) {
      const float cp = x_mul(cc, ivp), cs = x_mul(cc, ivs), u = x_mul(cp, cp), v = x_mul(cs, cs);
      const float p = sqrtf(x_add(1.f, -u)), sh = sqrtf(x_add(1.f, -v)), R = x_mul(p, sh);
      const float loss = x_fma(x_add(1.f, -u), v, u) / x_add(1.f, R), g = 2.f / v;
      const float d1 = x_fma(-g, loss, 1.f);
      lane_of(e[0], i) = x_mul(rh2, x_fma(-g, x_add(1.f, d1), 1.f));
      lane_of(e[1], i) = x_mul(x_mul(-rh, kk), p);
      lane_of(e[2], i) = x_mul(-rh, d1);
      lane_of(e[3], i) = x_mul(x_mul(rh, kk), sh);
      lane_of(e[4], i) = x_mul(lane_of(k2, i), loss);
    }
  }
}

// Rayleigh secular value, shape feature and base-2 log-magnitude of one (R1) or
// two (R2) samples of one trace at frequency w: the single-precision path of
// rayleigh_multi, explicitly rounded.  c holds the samples' velocities w / k.
template <class P>
__device__ __forceinline__ void rayleigh_eval32(const LayerView<float> &m, typename P::V k, typename P::V c, float w,
                                                typename P::V *F, typename P::V *shape, typename P::V *lmag) {
  using V = typename P::V;
  constexpr int NL = P::NL;
  const float tiny = 1e-30f;
  const float iw = 1.f / w, iw2 = x_mul(iw, iw);
  const int last = m.L - 1;
  const V k2 = P::mul(k, k);
  V e[5];
  start32<P>(e, k, k2, c, w, iw2, m.ivp(last), m.ivs(last), m.vs2(last), m.rho(last));
  int ex[NL];
  V ev = P::splat(0.f);
#pragma unroll
  for (int i = 0; i < NL; ++i) {
    float t[5] = {lane_of(e[0], i), lane_of(e[1], i), lane_of(e[2], i), lane_of(e[3], i), lane_of(e[4], i)};
    ex[i] = scale_vector(t, 5, tiny);
#pragma unroll
    for (int j = 0; j < 5; ++j) lane_of(e[j], i) = t[j];
  }
  for (int l = m.L - 2; l >= m.water; --l) {
    const float h = m.h(l), ivp = m.ivp(l), vs2 = m.vs2(l), ivs = m.ivs(l), rho = m.rho(l), irho = m.irho(l);
    const float ka = x_mul(w, ivp), kb = x_mul(w, ivs), gammk = x_mul(x_mul(iw2, vs2), 2.f);
    const float rho2 = x_mul(rho, rho), irho2 = x_mul(irho, irho);
    bool evan[NL], any = false, all = true;
#pragma unroll
    for (int i = 0; i < NL; ++i) {
      evan[i] = x_mul(x_mul(MD200_EVANESCENT_RATIO, lane_of(c, i)), ivs) < 1.f;
      any |= evan[i];
      all &= evan[i];
    }
    V en[5] = {e[0], e[1], e[2], e[3], e[4]};
    V expo = P::splat(0.f);
    if constexpr (NL == 1) {
      if (evan[0]) expo = evanescent32(en, k, k2, c, h, ivp, ivs, rho, irho, rho2, irho2);
      else expo = step32<P>(en, k, k2, ka, kb, gammk, h, rho, irho, rho2, irho2);
    } else {
      if (!all) expo = step32<P>(en, k, k2, ka, kb, gammk, h, rho, irho, rho2, irho2);
      if (any) {
#pragma unroll
        for (int i = 0; i < NL; ++i) {
          if (evan[i]) {
            float t[5] = {lane_of(e[0], i), lane_of(e[1], i), lane_of(e[2], i), lane_of(e[3], i),
                          lane_of(e[4], i)};
            lane_of(expo, i) = evanescent32(t, lane_of(k, i), lane_of(k2, i), lane_of(c, i), h, ivp, ivs, rho,
                                            irho, rho2, irho2);
#pragma unroll
            for (int j = 0; j < 5; ++j) lane_of(en[j], i) = t[j];
          }
        }
      }
    }
    ev = P::add(ev, expo);
#pragma unroll
    for (int i = 0; i < NL; ++i) {
      float t[5] = {lane_of(en[0], i), lane_of(en[1], i), lane_of(en[2], i), lane_of(en[3], i), lane_of(en[4], i)};
      ex[i] += scale_vector(t, 5, tiny);
#pragma unroll
      for (int j = 0; j < 5; ++j) lane_of(e[j], i) = t[j];
    }
  }
  V lm;
#pragma unroll
  for (int i = 0; i < NL; ++i) lane_of(lm, i) = static_cast<float>(ex[i]);
  lm = P::fma(ev, P::splat(1.4426950408889634f), lm);
  if (m.water) {
    const float h0 = m.h(0), ivp0 = m.ivp(0), rho0 = m.rho(0), ka = x_mul(w, ivp0);
#pragma unroll
    for (int i = 0; i < NL; ++i) {
      const float kk = lane_of(k, i);
      const float X = x_mul(x_add(kk, ka), fabsf(x_add(kk, -ka)));
      const float irf = R1::rsqrt0(X), rf = x_mul(X, irf), ph = x_mul(rf, h0);
      float cpw, wv;
      if (kk < ka) {
        float sn;
        sincos32<R1>(ph, &sn, &cpw);
        wv = x_mul(sn, irf);
      } else if (kk == ka) {
        cpw = 1.f;
        wv = h0;
      } else {
        const float ez = __expf(-ph), z = x_mul(ez, ez);
        cpw = x_fma(z, .5f, .5f);
        wv = x_mul(x_fma(z, -.5f, .5f), irf);
      }
      float pair[2] = {x_mul(cpw, lane_of(e[0], i)), x_mul(x_mul(wv, lane_of(e[1], i)), rho0)};
      const int pex = scale_vector(pair, 2, tiny);
      const float u = pair[0], v = pair[1], nn = x_add(x_fma(v, v, x_mul(u, u)), tiny), Fv = x_add(u, -v);
      if (shape) lane_of(*shape, i) = x_mul(Fv, rsqrtf(nn));
      if (lmag) lane_of(*lmag, i) = x_add(lane_of(lm, i), x_fma(.5f, log2f(nn), static_cast<float>(pex)));
      lane_of(*F, i) = Fv;
    }
  } else {
    const V n2 = P::add(P::fma(e[4], e[4], P::fma(e[3], e[3], P::fma(e[2], e[2], P::fma(e[1], e[1],
                                                                                     P::mul(e[0], e[0]))))),
                        P::splat(tiny));
#pragma unroll
    for (int i = 0; i < NL; ++i) {
      const float nn = lane_of(n2, i);
      if (shape) lane_of(*shape, i) = x_mul(lane_of(e[0], i), rsqrtf(nn));
      if (lmag) lane_of(*lmag, i) = x_fma(.5f, log2f(nn), lane_of(lm, i));
    }
    *F = e[0];
  }
}
// Rayleigh secular values F(k_s, w) of S samples at one frequency, with shape
// features g = F / |e| (water top: the fluid form).  Units: k = w / c in rad/km,
// w in rad/s.  The S recurrences are independent and interleaved layer by layer
// (instruction-level parallelism for latency-bound single-precision scans).
// With `lmag`, also the base-2 logarithm of the magnitude |e| of the
// unnormalised vector: it is smooth across ordinary roots and dips
// logarithmically where the whole vector nearly vanishes, the signature of a
// close root pair.  With `levan`, the part of that logarithm the evanescent
// scaling factored out (base 2 of exp(sum r h)).  With `fmax` (solid models),
// F on the scale of a recurrence renormalised to max |e_i| = 1 after every
// layer: F / max |e_i| of the final vector, |value| <= 1.
template <class N, class T, int S>
MD200_FN void rayleigh_multi(const LayerView<T> &m, const N *k, const N &w, N *F, N *shape,
                             typename Base<N>::type *lmag, typename Base<N>::type *levan = nullptr,
                             typename Base<N>::type *fmax = nullptr) {
  using B = typename Base<N>::type;
#if defined(__CUDA_ARCH__)
  // the scan's single-precision evaluations: explicitly rounded (rayleigh_eval32)
  if constexpr (std::is_same<N, float>::value && std::is_same<T, float>::value && S == 1) {
    if (levan == nullptr && fmax == nullptr) {
      rayleigh_eval32<R1>(m, k[0], w / k[0], w, F, shape, lmag);
      return;
    }
  }
#endif
  const B tiny = sizeof(B) == 4 ? B(1e-30) : B(1e-40);
  const N iw = lift_one<N>() / w;
  const N iw2 = iw * iw;
  const int last = m.L - 1;
  N e[S][5], k2[S];
  int ex[S];
  B ev[S];
#pragma unroll
  for (int s = 0; s < S; ++s) {
    k2[s] = k[s] * k[s];
    const T rh = m.rho(last);
    rayleigh_start<N, T>(e[s], k[s], k2[s], w, iw2, m.ivp(last), m.ivs(last), m.vs2(last), rh);
    if constexpr (sizeof(N) == sizeof(float)) {
      // single precision: the factored start vector well below the shear velocity
      const float c = w / k[s];
      const float ivs_l = m.ivs(last);
      if (MD200_EVANESCENT_RATIO * c * ivs_l < 1.f) {
        const float cp = c * m.ivp(last), cs = c * ivs_l, u = cp * cp, v = cs * cs;
        const float p = sqrtf(1.f - u), sh = sqrtf(1.f - v), R = p * sh;
        const float loss = (u + (1.f - u) * v) / (1.f + R), g = 2.f / v;
        const float d1 = 1.f - g * loss;
        e[s][0] = rh * rh * (1.f - g * (1.f + d1));
        e[s][1] = -rh * k[s] * p;
        e[s][2] = -rh * d1;
        e[s][3] = rh * k[s] * sh;
        e[s][4] = k2[s] * loss;
      }
    }
    ex[s] = scale_vector(e[s], 5, tiny);
    ev[s] = B(0);
  }
  for (int l = m.L - 2; l >= m.water; --l) {
    const T h = m.h(l), ivp = m.ivp(l), vs2 = m.vs2(l), ivs = m.ivs(l), rho = m.rho(l), irho = m.irho(l);
#pragma unroll
    for (int s = 0; s < S; ++s) {
      if constexpr (sizeof(N) == sizeof(float)) {
        const float c = w / k[s];
        if (MD200_EVANESCENT_RATIO * c * ivs < 1.f)
          ev[s] += rayleigh_layer_evanescent(e[s], k[s], k2[s], c, h, ivp, ivs, rho, irho);
        else
          ev[s] += rayleigh_layer_f32(e[s], k[s], k2[s], w, iw2, h, ivp, vs2, ivs, rho, irho);
      } else {
        ev[s] += rayleigh_layer(e[s], k[s], k2[s], w, iw2, h, ivp, vs2, ivs, rho, irho);
      }
      ex[s] += scale_vector(e[s], 5, tiny);
    }
  }
#pragma unroll
  for (int s = 0; s < S; ++s) {
    if (lmag) lmag[s] = static_cast<B>(ex[s]) + ev[s] * B(1.4426950408889634);
    if (levan) levan[s] = ev[s] * B(1.4426950408889634);
    if (m.water) {
      N cp, wv;
      water_top<N, T>(k[s], w, m.h(0), m.ivp(0), &cp, &wv);
      const N t0 = cp * e[s][0], t1 = wv * e[s][1] * m.rho(0);
      N pair[2] = {t0, t1};
      const int pex = scale_vector(pair, 2, tiny);
      const N u = pair[0], v = pair[1];
      if (shape) shape[s] = (u - v) * m_rsqrt(u * u + v * v + lift_one<N>() * tiny);
      if (lmag) lmag[s] += static_cast<B>(pex) + B(0.5) * m_log2(val(u * u + v * v) + tiny);
      F[s] = u - v;
    } else {
      const N norm2 = e[s][0] * e[s][0] + e[s][1] * e[s][1] + e[s][2] * e[s][2] + e[s][3] * e[s][3] +
                      e[s][4] * e[s][4];
      if (shape) shape[s] = e[s][0] * m_rsqrt(norm2 + lift_one<N>() * tiny);
      if (lmag) lmag[s] += B(0.5) * m_log2(val(norm2) + tiny);
      if (fmax) {
        B big = B(0);
#pragma unroll
        for (int i = 0; i < 5; ++i) big = m_max(big, m_abs(val(e[s][i])));
        fmax[s] = big > B(0) ? val(e[s][0]) / big : val(e[s][0]);
      }
      F[s] = e[s][0];
    }
  }
}

template <class N, class T>
MD200_FN N rayleigh_secular(const LayerView<T> &m, const N &k, const N &w, N *shape,
                            typename Base<N>::type *lmag = nullptr, typename Base<N>::type *levan = nullptr) {
  N F;
  rayleigh_multi<N, T, 1>(m, &k, w, &F, shape, lmag, levan);
  return F;
}

// Entries of one SH layer step, [[cq, z mu], [y / mu, cq]]: the S-wave block of
// wavenumber k against the layer's shear wavenumber kj; returns the exponent the
// scaled hyperbolic functions factor out (value part).
template <class N, class T>
MD200_FN typename Base<N>::type love_entries(const N &k, const N &kj, T h, N *cq, N *y, N *z) {
  N scale;
  return wave_block<N, T>(k, kj, h, cq, y, z, &scale);
}

// Love secular values (SH propagator) and shape features of S samples.
template <class N, class T, int S>
MD200_FN void love_multi(const LayerView<T> &m, const N *k, const N &w, N *F, N *shape,
                         typename Base<N>::type *lmag, typename Base<N>::type *levan = nullptr) {
  using B = typename Base<N>::type;
  const B tiny = sizeof(B) == 4 ? B(1e-30) : B(1e-40);
  const int last = m.L - 1;
  N e[S][2];
  int ex[S];
  B ev[S];
#pragma unroll
  for (int s = 0; s < S; ++s) {
    const N kb = w * m.ivs(last);
    N r, ir;
    radical(k[s], kb, &r, &ir);
    e[s][0] = r * m.rho(last);
    e[s][1] = lift_one<N>() * (m.ivs(last) * m.ivs(last));
    ex[s] = 0;
    ev[s] = B(0);
  }
  auto layer = [&](int j) {
    const T h = m.h(j), mu = m.rho(j) * m.vs2(j), imu = m.imu(j), ivs = m.ivs(j);
#pragma unroll
    for (int s = 0; s < S; ++s) {
      const N kj = w * ivs;
      N cq, y, z;
      if constexpr (sizeof(N) == sizeof(float)) {
        // branch-free single precision: both forms, selected
        N r, ir;
        radical(k[s], kj, &r, &ir);
        const float q = r * h;
        float sn, cs;
        m_sincos(q, &sn, &cs);
        const float eq = m_exp(-q), f = eq * eq;
        const bool prop = k[s] < kj;
        cq = prop ? cs : .5f * (1.f + f);
        const float half = prop ? sn : .5f * (1.f - f);
        y = ir > 0.f ? half * ir : h;
        z = prop ? -(r * half) : r * half;
        ev[s] += prop ? 0.f : q;
      } else {
        ev[s] += love_entries<N, T>(k[s], kj, h, &cq, &y, &z);
      }
      const N u = e[s][0] * cq + e[s][1] * z * mu;
      const N v = e[s][0] * y * imu + e[s][1] * cq;
      e[s][0] = u;
      e[s][1] = v;
      ex[s] += scale_vector(e[s], 2, tiny);
    }
  };
  if constexpr (sizeof(N) == sizeof(float)) {
    // two layers per iteration: the next layer's special functions overlap this
    // one's recurrence (measured 5 % faster for the FP32 Love scan, 9 % slower
    // for the FP64 one, whose longer body already fills the pipes)
#pragma unroll 2
    for (int j = last - 1; j >= m.water; --j) layer(j);
  } else {
    for (int j = last - 1; j >= m.water; --j) layer(j);
  }
#pragma unroll
  for (int s = 0; s < S; ++s) {
    const N norm2 = e[s][0] * e[s][0] + e[s][1] * e[s][1];
    if (shape) shape[s] = e[s][0] * m_rsqrt(norm2 + lift_one<N>() * tiny);
    if (lmag)
      lmag[s] = static_cast<B>(ex[s]) + ev[s] * B(1.4426950408889634) + B(0.5) * m_log2(val(norm2) + tiny);
    if (levan) levan[s] = ev[s] * B(1.4426950408889634);
    F[s] = e[s][0];
  }
}

template <class N, class T>
MD200_FN N love_secular(const LayerView<T> &m, const N &k, const N &w, N *shape,
                        typename Base<N>::type *lmag = nullptr, typename Base<N>::type *levan = nullptr) {
  N F;
  love_multi<N, T, 1>(m, &k, w, &F, shape, lmag, levan);
  return F;
}

// S samples at once (WAVE: 0 Rayleigh, 1 Love).
template <class N, class T, int S, int WAVE>
MD200_FN void secular_multi(const LayerView<T> &m, const N *k, const N &w, N *F, N *shape,
                            typename Base<N>::type *lmag) {
  if constexpr (WAVE) love_multi<N, T, S>(m, k, w, F, shape, lmag);
  else rayleigh_multi<N, T, S>(m, k, w, F, shape, lmag);
}

template <class N, class T>
MD200_FN N secular(const LayerView<T> &m, int wave, const N &k, const N &w, N *shape,
                   typename Base<N>::type *lmag = nullptr, typename Base<N>::type *levan = nullptr) {
  return wave ? love_secular<N, T>(m, k, w, shape, lmag, levan) : rayleigh_secular<N, T>(m, k, w, shape, lmag, levan);
}

}  // namespace md200
