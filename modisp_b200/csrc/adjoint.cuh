// adjoint.cuh -- phase- and group-velocity Jacobians of the roots with respect
// to every layer's thickness, Vp, Vs and density (no counterpart in the
// reference, which has no derivatives of its roots).
//
// At a root F(k, omega; m) = 0 of the secular function (k = omega / c):
//   dk/dm = -F_m / F_k,   dc/dm = (c / k) F_m / F_k,
//   U = -F_k / F_omega,   dU/dm = dU/dm|_k + dU/dk|_m dk/dm with
//   dU/dm|_k = -(F_km F_w - F_k F_wm) / F_w^2,  dU/dk|_m = -(F_kk F_w - F_k F_wk) / F_w^2.
// The engine's F is the reference function times a smooth positive factor (the
// per-layer power-of-two scales, held fixed, and the exp(-(P+Q)) of the scaled
// hyperbolic functions); each expression above is a ratio that the factor
// leaves unchanged on the root curve, so the Jacobians are those of the
// reference function.
//
// Per root (one thread), all arithmetic on D2 = (value, d/dk, d/domega) numbers:
//  1. forward sweep with an extra k-direction on top of D2: F, F_k, F_w, F_kk,
//     F_kw; the per-layer scale exponents are recorded and the D2 state vector
//     is checkpointed every JAC_SEG layers;
//  2. reverse sweep, top to bottom: each segment's states are recomputed from
//     its checkpoint (the layer matrices are recomputed, never stored), and the
//     hand-written adjoint of the layer step -- the transposed compound matrix
//     for the adjoint vector, then reverse accumulation through the 15 entry
//     polynomials into the wave blocks and the material constants -- yields the
//     row's derivatives of (F, F_k, F_w): the D2 parts of the adjoint carry the
//     (k, omega) derivatives of the parameter gradient (forward-over-reverse).
#pragma once
#include "engine.cuh"
#include "secular.cuh"

#ifdef MD200_HOST_SECULAR
#define MD200_HD __host__ __device__
#define MD200_OUTLINE __host__ __device__
#else
#define MD200_HD __device__
// the layer steps of the Jacobian sweeps are called, not inlined: each gets the
// whole register file instead of competing with the sweep's bookkeeping
#define MD200_OUTLINE __device__ __noinline__
#endif

namespace md200 {

using D2 = Dual<double, 2>;  // value, d/dk, d/domega
using K1 = Dual<D2, 1>;      // ... and d/dk of all three (second order in k)
using Q2 = Dual<D2, 2>;      // d/d(h, 1/v) of one wave block
using P4 = Dual<D2, 4>;      // d/d(h, vp, vs, rho) of one row (start vector, fluid top)

constexpr int JAC_SEG = 12;     // layer steps per recomputed segment
constexpr int JAC_MAXSEG = 22;  // checkpoints: up to 264 layer steps (the API's 256 rows fit)
constexpr int JAC_MAX_STEPS = JAC_SEG * JAC_MAXSEG;

MD200_FN P4 lift4(const D2 &x) {
  P4 r;
  r.v = x;
#pragma unroll
  for (int i = 0; i < 4; ++i) r.d[i] = D2(0);
  return r;
}
// A layer constant x with derivative `slope` along parameter direction `dir`.
MD200_FN P4 seed4(double x, int dir, double slope) {
  P4 r(x);
  r.d[dir] = D2(slope);
  return r;
}
MD200_FN double pow2(int e) { return scalbn(1.0, e); }

// A row's constants as nested duals in its own (h, vp, vs, rho).
struct RowP4 {
  P4 h, ivp, ivs, vs2, rho, irho;
};
MD200_FN RowP4 row_p4(const double *tab, int Ls, int j) {
  const double h = tab[j], ivp = tab[Ls + j], ivs = tab[2 * Ls + j], vs2 = tab[3 * Ls + j];
  const double rho = tab[4 * Ls + j], irho = tab[5 * Ls + j], vs = tab[8 * Ls + j];
  RowP4 r;
  r.h = seed4(h, 0, 1.);
  r.ivp = seed4(ivp, 1, -ivp * ivp);
  r.ivs = vs > 0. ? seed4(ivs, 2, -ivs * ivs) : P4(0.);
  r.vs2 = seed4(vs2, 2, 2. * vs);
  r.rho = seed4(rho, 3, 1.);
  r.irho = seed4(irho, 3, -irho * irho);
  return r;
}

// One wave block with its derivatives along (h, 1/v): cs, sr, rs, scale.
struct BlockQ {
  Q2 cs, sr, rs, sc;
};
MD200_FN void block_q(const D2 &k, const D2 &w, double h, double iv, BlockQ &b) {
  Q2 kq, wq, hq(h), ivq(iv);
  kq.v = k;
  kq.d[0] = kq.d[1] = D2(0);
  wq.v = w;
  wq.d[0] = wq.d[1] = D2(0);
  hq.d[0] = D2(1);
  ivq.d[1] = D2(1);
  const Q2 kv = wq * ivq;
  wave_block<Q2, Q2>(kq, kv, hq, &b.cs, &b.sr, &b.rs, &b.sc);
}

// Derivatives of (F, F_k, F_w) along one row's parameters, as D2 numbers
// (value: F_m; d[0]: F_km; d[1]: F_wm), for m = h, vp, vs, rho.
struct RowGrad {
  D2 g[4];
};

// Reverse step through one Rayleigh layer.  s: the state before the step; lam:
// the adjoint of the (scaled) state after it, replaced by the adjoint of s;
// r: the step's power-of-two scale.  Returns the row's derivatives.
MD200_OUTLINE RowGrad rayleigh_layer_adjoint(const D2 &k, const D2 &k2, const D2 &w, const D2 &iw2, double h,
                                             double ivp, double ivs, double vs2, double vs, double rho,
                                             double irho, const D2 s[5], D2 lam[5], double r) {
  BlockQ P, S;
  block_q(k, w, h, ivp, P);
  block_q(k, w, h, ivs, S);
  const D2 cosp = P.cs.v, wv = P.sr.v, xv = P.rs.v, a0p = P.sc.v;
  const D2 cosq = S.cs.v, yv = S.sr.v, zv = S.rs.v, a0s = S.sc.v;
  const D2 a0 = a0p * a0s;
  const D2 gammk = (iw2 * vs2) * 2.;
  const D2 gam = gammk * k2;
  RayleighEntries<D2> X;
  rayleigh_poly<D2, double>(X, cosp, wv, xv, cosq, yv, zv, a0, gam, gammk, k2, rho, irho);

  // adjoint of M s, scaled: W_X = sum over the positions of entry X of lam_row s_col
  D2 lr[5];
  for (int i = 0; i < 5; ++i) lr[i] = lam[i] * r;
  const D2 t = k2 * -2.;
  const D2 s2t = s[2] * t;
  const D2 WA = lr[0] * s[0] + lr[4] * s[4], WE = lr[0] * s[1] + lr[3] * s[4];
  const D2 WJ = lr[0] * s2t + lr[2] * s[4], WF = lr[0] * s[3] + lr[1] * s[4];
  const D2 WO = lr[0] * s[4], WD = lr[1] * s[0] + lr[4] * s[3], WB = lr[1] * s[1] + lr[3] * s[3];
  const D2 WH = lr[1] * s2t + lr[2] * s[3], WN = lr[1] * s[3], WI = lr[2] * s[0] + lr[4] * s2t;
  const D2 WG = lr[2] * s[1] + lr[3] * s2t, WK = lr[2] * s[2], WC = lr[3] * s[0] + lr[4] * s[1];
  const D2 WM = lr[3] * s[1], WL = lr[4] * s[0];

  // adjoint vector through the transposed matrix
  const D2 tcol = X.J * lr[0] + X.H * lr[1] + X.G * lr[3] + X.I * lr[4];
  lam[0] = X.A * lr[0] + X.D * lr[1] + X.I * lr[2] + X.C * lr[3] + X.Lm * lr[4];
  lam[1] = X.E * lr[0] + X.B * lr[1] + X.G * lr[2] + X.M * lr[3] + X.C * lr[4];
  lam[2] = t * tcol + X.K * lr[2];
  lam[3] = X.F * lr[0] + X.Nn * lr[1] + X.H * lr[2] + X.B * lr[3] + X.D * lr[4];
  lam[4] = X.O * lr[0] + X.F * lr[1] + X.J * lr[2] + X.E * lr[3] + X.A * lr[4];

  // density: each entry is rho^n times a density-free polynomial
  const D2 brho = ((X.E * WE + X.F * WF + X.J * WJ) + X.O * WO * 2. - (X.D * WD + X.I * WI + X.C * WC) -
                   X.Lm * WL * 2.) * irho;

  // reverse through the entry polynomials
  const D2 cpcq = cosp * cosq, cpy = cosp * yv, cpz = cosp * zv, cqw = cosq * wv, cqx = cosq * xv;
  const D2 xy = xv * yv, xz = xv * zv, wy = wv * yv, wz = wv * zv;
  const D2 gm1 = gam - 1., twgm1 = gam + gm1, gmgmk = gam * gammk, gmgm1 = gam * gm1, gm1sq = gm1 * gm1;
  const D2 a0pq = a0 - cpcq;
  const double rho2 = rho * rho, irho2 = irho * irho;
  const D2 z0(0);
  const D2 bA = WA - WK * 2.;  // K = a0 + 2 cpcq - 2 A
  D2 b_a0 = WK, b_cpcq = WK * 2. + WB + bA;
  D2 b_gmgm1 = -(a0pq * bA) * 2., b_a0pq = -(gmgm1 * bA) * 2., b_gmgmk = -(xz * bA), b_xz = -(gmgmk * bA);
  D2 b_gm1sq = -(k2 * wy * bA), b_wy = -(k2 * gm1sq * bA);
  D2 b_cpy = z0, b_cqx = z0, b_twgm1 = z0, b_gammk = z0, b_gm1 = z0, b_cpz = z0, b_cqw = z0, b_gam = z0;
  {  // D = (k2 cpy - cqx) / rho
    const D2 d = WD * irho;
    b_cpy = b_cpy + k2 * d;
    b_cqx = b_cqx - d;
  }
  {  // I = -(twgm1 a0pq + gammk xz + k2 gm1 wy) / rho
    const D2 d = -(WI * irho);
    b_twgm1 = b_twgm1 + a0pq * d;
    b_a0pq = b_a0pq + twgm1 * d;
    b_gammk = b_gammk + xz * d;
    b_xz = b_xz + gammk * d;
    b_gm1 = b_gm1 + k2 * wy * d;
    b_wy = b_wy + k2 * gm1 * d;
  }
  {  // C = (cpz - k2 cqw) / rho
    const D2 d = WC * irho;
    b_cpz = b_cpz + d;
    b_cqw = b_cqw - k2 * d;
  }
  {  // Lm = -(2 k2 a0pq + xz + k2^2 wy) / rho^2
    const D2 d = -(WL * irho2);
    b_a0pq = b_a0pq + k2 * d * 2.;
    b_xz = b_xz + d;
    b_wy = b_wy + k2 * k2 * d;
  }
  {  // E = (gmgmk cpz - gm1sq cqw) rho
    const D2 d = WE * rho;
    b_gmgmk = b_gmgmk + cpz * d;
    b_cpz = b_cpz + gmgmk * d;
    b_gm1sq = b_gm1sq - cqw * d;
    b_cqw = b_cqw - gm1sq * d;
  }
  {  // G = gammk cpz - gm1 cqw
    b_gammk = b_gammk + cpz * WG;
    b_cpz = b_cpz + gammk * WG;
    b_gm1 = b_gm1 - cqw * WG;
    b_cqw = b_cqw - gm1 * WG;
  }
  const D2 b_wz = -WM, b_xy = -WN;  // M = -wz, Nn = -xy
  {  // F = (gm1sq cpy - gmgmk cqx) rho
    const D2 d = WF * rho;
    b_gm1sq = b_gm1sq + cpy * d;
    b_cpy = b_cpy + gm1sq * d;
    b_gmgmk = b_gmgmk - cqx * d;
    b_cqx = b_cqx - gmgmk * d;
  }
  {  // H = gm1 cpy - gammk cqx
    b_gm1 = b_gm1 + cpy * WH;
    b_cpy = b_cpy + gm1 * WH;
    b_gammk = b_gammk - cqx * WH;
    b_cqx = b_cqx - gammk * WH;
  }
  {  // O = -(2 gmgmk gm1sq a0pq + gmgmk^2 xz + gm1sq^2 wy) rho^2
    const D2 d = -(WO * rho2);
    b_gmgmk = b_gmgmk + (gm1sq * a0pq + gmgmk * xz) * d * 2.;
    b_gm1sq = b_gm1sq + (gmgmk * a0pq + gm1sq * wy) * d * 2.;
    b_a0pq = b_a0pq + gmgmk * gm1sq * d * 2.;
    b_xz = b_xz + gmgmk * gmgmk * d;
    b_wy = b_wy + gm1sq * gm1sq * d;
  }
  {  // J = -(gammk gm1 twgm1 a0pq + gam gammk^2 xz + gm1 gm1sq wy) rho
    const D2 d = -(WJ * rho);
    b_gammk = b_gammk + (gm1 * twgm1 * a0pq + gam * gammk * xz * 2.) * d;
    b_gm1 = b_gm1 + (gammk * twgm1 * a0pq + gm1sq * wy) * d;
    b_twgm1 = b_twgm1 + gammk * gm1 * a0pq * d;
    b_a0pq = b_a0pq + gammk * gm1 * twgm1 * d;
    b_gam = b_gam + gammk * gammk * xz * d;
    b_xz = b_xz + gam * gammk * gammk * d;
    b_gm1sq = b_gm1sq + gm1 * wy * d;
    b_wy = b_wy + gm1 * gm1sq * d;
  }
  // intermediates, in reverse order of their definitions
  b_a0 = b_a0 + b_a0pq;
  b_cpcq = b_cpcq - b_a0pq;
  b_gm1 = b_gm1 + gm1 * b_gm1sq * 2.;
  b_gam = b_gam + gm1 * b_gmgm1 + gammk * b_gmgmk + b_twgm1;
  b_gm1 = b_gm1 + gam * b_gmgm1 + b_twgm1;
  b_gammk = b_gammk + gam * b_gmgmk;
  b_gam = b_gam + b_gm1;
  b_gammk = b_gammk + k2 * b_gam;
  const D2 b_vs2 = iw2 * b_gammk * 2.;
  // products of the wave blocks
  const D2 b_cosp = b_cpcq * cosq + b_cpy * yv + b_cpz * zv;
  const D2 b_cosq = b_cpcq * cosp + b_cqw * wv + b_cqx * xv;
  const D2 b_wv = b_cqw * cosq + b_wy * yv + b_wz * zv;
  const D2 b_xv = b_cqx * cosq + b_xy * yv + b_xz * zv;
  const D2 b_yv = b_cpy * cosp + b_xy * xv + b_wy * wv;
  const D2 b_zv = b_cpz * cosp + b_xz * xv + b_wz * wv;
  const D2 b_a0p = b_a0 * a0s, b_a0s = b_a0 * a0p;
  RowGrad g;
  D2 cp[2], cs[2];
  for (int q = 0; q < 2; ++q) {
    cp[q] = b_cosp * P.cs.d[q] + b_wv * P.sr.d[q] + b_xv * P.rs.d[q] + b_a0p * P.sc.d[q];
    cs[q] = b_cosq * S.cs.d[q] + b_yv * S.sr.d[q] + b_zv * S.rs.d[q] + b_a0s * S.sc.d[q];
  }
  g.g[0] = cp[0] + cs[0];
  g.g[1] = cp[1] * (-ivp * ivp);
  g.g[2] = cs[1] * (-ivs * ivs) + b_vs2 * (2. * vs);
  g.g[3] = brho;
  return g;
}

// Reverse step through one SH layer (u = e0 cq + e1 z mu, v = e0 y / mu + e1 cq).
MD200_OUTLINE RowGrad love_layer_adjoint(const D2 &k, const D2 &w, double h, double ivs, double vs, double rho,
                                         double vs2, double imu, const D2 s[2], D2 lam[2], double r) {
  BlockQ S;
  block_q(k, w, h, ivs, S);
  const D2 cq = S.cs.v, y = S.sr.v, z = S.rs.v;
  const double mu = rho * vs2;
  const D2 l0 = lam[0] * r, l1 = lam[1] * r;
  lam[0] = l0 * cq + l1 * (y * imu);
  lam[1] = l0 * (z * mu) + l1 * cq;
  const D2 b_cq = l0 * s[0] + l1 * s[1], b_z = l0 * s[1] * mu, b_y = l1 * s[0] * imu;
  const D2 b_mu = l0 * s[1] * z, b_imu = l1 * s[0] * y;
  D2 c[2];
  for (int q = 0; q < 2; ++q) c[q] = b_cq * S.cs.d[q] + b_y * S.sr.d[q] + b_z * S.rs.d[q];
  RowGrad g;
  g.g[0] = c[0];
  g.g[1] = D2(0);
  g.g[2] = c[1] * (-ivs * ivs) + b_mu * (2. * rho * vs) + b_imu * (-2. * imu / vs);
  g.g[3] = b_mu * vs2 + b_imu * (-imu / rho);
  return g;
}

// Forward layer steps of the Jacobian sweeps (out of line).
MD200_OUTLINE int rayleigh_step_k1(K1 e[5], const K1 &k, const K1 &k2, const K1 &w, const K1 &iw2, double h,
                                   double ivp, double vs2, double ivs, double rho, double irho) {
  rayleigh_layer<K1, double>(e, k, k2, w, iw2, h, ivp, vs2, ivs, rho, irho);
  return scale_vector(e, 5, 1e-40);
}
MD200_OUTLINE void rayleigh_step_d2(D2 e[5], const D2 &k, const D2 &k2, const D2 &w, const D2 &iw2, double h,
                                    double ivp, double vs2, double ivs, double rho, double irho, double r) {
  rayleigh_layer<D2, double>(e, k, k2, w, iw2, h, ivp, vs2, ivs, rho, irho);
  for (int i = 0; i < 5; ++i) e[i] = e[i] * r;
}

// Per-root quantities of the forward sweep.
struct RootForward {
  double Fk, Fw, Fkk, Fkw;
};

// Forward + reverse sweeps for one root; `sink(row, grad)` receives each
// compact row's parameter derivatives (top row first, half-space last).
template <int WAVE, class Sink>
MD200_HD bool root_adjoint(const LayerView<double> &m, const double *tab, double w, double c,
                           RootForward &fw, Sink &&sink) {
  const int L = m.L, Ls = m.Ls, last = L - 1, top = m.water;
  const int nsteps = last - top;  // layer steps (rows last-1 .. top)
  if (nsteps > JAC_MAX_STEPS) return false;
  const double tiny = 1e-40;
  constexpr int NV = WAVE ? 2 : 5;
  // (k, omega) duals and their k-lifts
  D2 k, wd;
  k.v = w / c; k.d[0] = 1.; k.d[1] = 0.;
  wd.v = w; wd.d[0] = 0.; wd.d[1] = 1.;
  const D2 iw = D2(1) / wd, iw2 = iw * iw, k2 = k * k;
  K1 kk, ww;
  kk.v = k; kk.d[0] = D2(1);
  ww.v = wd; ww.d[0] = D2(0);
  const K1 iwx = K1(1) / ww, iw2x = iwx * iwx, k2x = kk * kk;

  D2 ck[JAC_MAXSEG][NV];
  short ex[JAC_MAX_STEPS];  // per-step binade exponents of a double, |e| < 1100
  int ex0 = 0, pex = 0;

  // ---- 1. forward sweep, exponents and checkpoints ----
  K1 e[NV];
  if constexpr (WAVE == 0) {
    rayleigh_start<K1, double>(e, kk, k2x, ww, iw2x, m.ivp(last), m.ivs(last), m.vs2(last), m.rho(last));
    ex0 = scale_vector(e, 5, tiny);
  } else {
    const K1 kb = ww * m.ivs(last);
    K1 r, ir;
    radical(kk, kb, &r, &ir);
    e[0] = r * m.rho(last);
    e[1] = K1(1) * (m.ivs(last) * m.ivs(last));
  }
  for (int s = 0; s < nsteps; ++s) {
    const int l = last - 1 - s;
    if (s % JAC_SEG == 0)
      for (int i = 0; i < NV; ++i) ck[s / JAC_SEG][i] = e[i].v;
    if constexpr (WAVE == 0) {
      ex[s] = (short)rayleigh_step_k1(e, kk, k2x, ww, iw2x, m.h(l), m.ivp(l), m.vs2(l), m.ivs(l), m.rho(l), m.irho(l));
    } else {
      const K1 kj = ww * m.ivs(l);
      K1 cq, y, z;
      love_entries<K1, double>(kk, kj, m.h(l), &cq, &y, &z);
      const double mu = m.rho(l) * m.vs2(l);
      const K1 u = e[0] * cq + e[1] * z * mu;
      const K1 v = e[0] * y * m.imu(l) + e[1] * cq;
      e[0] = u;
      e[1] = v;
      ex[s] = (short)scale_vector(e, NV, tiny);
    }
  }
  K1 F;
  if (WAVE == 0 && top) {
    K1 cpx, wvx;
    water_top<K1, double>(kk, ww, m.h(0), m.ivp(0), &cpx, &wvx);
    K1 pair[2] = {cpx * e[0], wvx * e[1] * m.rho(0)};
    pex = scale_vector(pair, 2, tiny);
    F = pair[0] - pair[1];
  } else {
    F = e[0];
  }
  fw.Fk = F.v.d[0];
  fw.Fw = F.v.d[1];
  fw.Fkk = F.d[0].d[0];
  fw.Fkw = F.d[0].d[1];
  if (!isfinite(fw.Fk) || !isfinite(fw.Fw) || fw.Fk == 0. || fw.Fw == 0.) return false;

  // ---- 2. reverse sweep ----
  D2 lam[NV];
  for (int i = 0; i < NV; ++i) lam[i] = D2(0);
  const P4 kP = lift4(k), k2P = lift4(k2), wP = lift4(wd), iw2P = lift4(iw2);
  if (WAVE == 0 && top) {
    // F = (cp e0 - wv e1 rho0) 2^-pex with the fluid row's own parameters
    const double rp = pow2(-pex);
    const RowP4 r0 = row_p4(tab, Ls, 0);
    P4 cp, wv;
    water_top<P4, P4>(kP, wP, r0.h, r0.ivp, &cp, &wv);
    const P4 Fw4 = (cp * lift4(e[0].v) - wv * lift4(e[1].v) * r0.rho) * rp;
    RowGrad g;
    for (int p = 0; p < 4; ++p) g.g[p] = Fw4.d[p];
    g.g[2] = D2(0);  // a fluid row has no shear velocity
    sink(0, g);
    lam[0] = cp.v * rp;
    lam[1] = -(wv.v * r0.rho.v) * rp;
  } else {
    lam[0] = D2(1);
  }
  const int nseg = (nsteps + JAC_SEG - 1) / JAC_SEG;
  D2 st[JAC_SEG][NV];
  for (int sg = nseg - 1; sg >= 0; --sg) {
    const int s0 = sg * JAC_SEG, s1 = nsteps < s0 + JAC_SEG ? nsteps : s0 + JAC_SEG;
    // recompute the segment's input states (stored exponents: the same scales)
    D2 x[NV];
    for (int i = 0; i < NV; ++i) x[i] = ck[sg][i];
    for (int s = s0; s < s1; ++s) {
      const int l = last - 1 - s;
      for (int i = 0; i < NV; ++i) st[s - s0][i] = x[i];
      if (s + 1 == s1) break;
      const double r = pow2(-ex[s]);
      if constexpr (WAVE == 0) {
        rayleigh_step_d2(x, k, k2, wd, iw2, m.h(l), m.ivp(l), m.vs2(l), m.ivs(l), m.rho(l), m.irho(l), r);
      } else {
        const D2 kj = wd * m.ivs(l);
        D2 cq, y, z;
        love_entries<D2, double>(k, kj, m.h(l), &cq, &y, &z);
        const double mu = m.rho(l) * m.vs2(l);
        const D2 u = x[0] * cq + x[1] * z * mu;
        const D2 v = x[0] * y * m.imu(l) + x[1] * cq;
        x[0] = u * r;
        x[1] = v * r;
      }
    }
    // reverse through the segment, top layer first
    for (int s = s1 - 1; s >= s0; --s) {
      const int l = last - 1 - s;
      const double r = pow2(-ex[s]);
      const double vs = tab[8 * Ls + l];
      RowGrad g;
      if constexpr (WAVE == 0)
        g = rayleigh_layer_adjoint(k, k2, wd, iw2, m.h(l), m.ivp(l), m.ivs(l), m.vs2(l), vs, m.rho(l), m.irho(l),
                                   st[s - s0], lam, r);
      else
        g = love_layer_adjoint(k, wd, m.h(l), m.ivs(l), vs, m.rho(l), m.vs2(l), m.imu(l), st[s - s0], lam, r);
      sink(l, g);
    }
  }
  // half-space: derivatives through the start vector
  {
    const RowP4 hs = row_p4(tab, Ls, last);
    RowGrad g;
    if constexpr (WAVE == 0) {
      P4 es[5];
      rayleigh_start<P4, P4>(es, kP, k2P, wP, iw2P, hs.ivp, hs.ivs, hs.vs2, hs.rho);
      const double r = pow2(-ex0);
      for (int p = 0; p < 4; ++p) {
        D2 acc = lam[0] * es[0].d[p];
        for (int i = 1; i < 5; ++i) acc = acc + lam[i] * es[i].d[p];
        g.g[p] = acc * r;
      }
    } else {
      const P4 kb = wP * hs.ivs;
      P4 r, ir;
      radical(kP, kb, &r, &ir);
      const P4 e0 = r * hs.rho, e1 = hs.ivs * hs.ivs;
      for (int p = 0; p < 4; ++p) g.g[p] = lam[0] * e0.d[p] + lam[1] * e1.d[p];
    }
    g.g[0] = D2(0);  // the half-space has no thickness
    sink(last, g);
  }
  return true;
}

#ifndef MD200_HOST_SECULAR
// ---------------------------------------------------------------------------
// root_jacobians: one thread per output cell (model, mode, period).
// Full mode (grad == nullptr): jac_c / jac_u [cell][4][Lmax] receive dc/dm and
// dU/dm (rows of zero thickness dropped by the engine keep 0; NaN where the
// root, or for jac_u the group velocity, is missing).
// Adjoint mode: grad [4][B][Lmax] += wc[cell] dc/dm + wu[cell] dU/dm.
// ---------------------------------------------------------------------------
template <int WAVE>
__global__ void __launch_bounds__(128) root_jacobians(Dev d, const double *vel, const double *grp, double *jac_c,
                                                      double *jac_u, const double *wc, const double *wu,
                                                      double *grad, int *nfail) {
  const int nm = d.nmodes, T = d.T, Lmax = d.Lmax;
  const long long ncell = static_cast<long long>(d.B) * nm * T;
  for (long long cell = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; cell < ncell;
       cell += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int b = static_cast<int>(cell / (static_cast<long long>(nm) * T));
    const int f = static_cast<int>(cell % T);
    const double c = vel[cell];
    const double U = grp ? grp[cell] : 0.;
    const bool want_u = jac_u != nullptr || (wu != nullptr && wu[cell] != 0.);
    double *jc = jac_c ? jac_c + cell * 4 * Lmax : nullptr;
    double *ju = jac_u ? jac_u + cell * 4 * Lmax : nullptr;
    const double wcc = wc ? wc[cell] : 0., wuc = wu ? wu[cell] : 0.;
    if (grad && wcc == 0. && wuc == 0.) continue;
    auto fill = [&](double *out, double x) {
      if (out)
        for (int i = 0; i < 4 * Lmax; ++i) out[i] = x;
    };
    if (!isfinite(c) || d.mstate[b] != 0) {
      fill(jc, NAN);
      fill(ju, NAN);
      continue;
    }
    const bool u_ok = !grp || isfinite(U);
    if (!u_ok) fill(ju, NAN);
    const LayerView<double> m = global_view(d, b);
    const double *tab = layer_table<double>(d, b);
    const double w = TWO_PI / d.periods[f];
    const double k = w / c;
    // compact row -> input row (rows kept by prep_models: the first, the last
    // and every row of positive thickness)
    const double *hin = d.h + static_cast<size_t>(b) * Lmax;
    int ci = 0, jo = 0;  // compact row ci is input row jo
    RootForward fwd{};
    auto sink = [&](int row, const RowGrad &g) {
      // rows arrive in increasing order: advance to the input row of `row`
      while (ci < row && jo < Lmax - 1) {
        ++jo;
        while (jo < Lmax - 1 && !(hin[jo] > 0.)) ++jo;
        ++ci;
      }
      for (int p = 0; p < 4; ++p) {
        const double Fm = g.g[p].v, Fkm = g.g[p].d[0], Fwm = g.g[p].d[1];
        const double dk = -Fm / fwd.Fk;
        const double dc = -(c / k) * dk;
        double du = 0.;
        if (want_u && u_ok) {
          const double iw2 = 1. / (fwd.Fw * fwd.Fw);
          const double dudm = -(Fkm * fwd.Fw - fwd.Fk * Fwm) * iw2;
          const double dudk = -(fwd.Fkk * fwd.Fw - fwd.Fk * fwd.Fkw) * iw2;
          du = dudm + dudk * dk;
        }
        const size_t at = static_cast<size_t>(p) * Lmax + jo;
        if (grad) {
          const double contrib = wcc * dc + (u_ok ? wuc * du : 0.);
          if (contrib != 0.) atomicAdd(grad + (static_cast<size_t>(p) * d.B + b) * Lmax + jo, contrib);
        } else {
          jc[at] = dc;
          if (ju && u_ok) ju[at] = du;
        }
      }
    };
    if (jc) fill(jc, 0.);
    if (ju && u_ok) fill(ju, 0.);
    const bool ok = root_adjoint<WAVE>(m, tab, w, c, fwd, sink);
    if (!ok) {
      fill(jc, NAN);
      fill(ju, NAN);
      if (nfail) atomicAdd(nfail, 1);
    }
  }
}
#endif  // MD200_HOST_SECULAR

}  // namespace md200
