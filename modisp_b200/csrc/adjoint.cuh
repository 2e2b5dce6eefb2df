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
// Per root (one thread):
//  1. forward sweep with second-order duals in (k, omega): F, F_k, F_w, F_kk,
//     F_kw; the per-layer scale exponents are recorded and the (k, omega)-dual
//     state vector is checkpointed every JAC_SEG layers;
//  2. reverse sweep, top to bottom: the layer's states are recomputed from the
//     checkpoint (the layer matrices are recomputed, never stored), the adjoint
//     vector runs through the transposed layer matrix, and the layer's four
//     parameter derivatives of (F, F_k, F_w) come from the layer matrix in
//     nested duals (outer: h, vp, vs, rho of this row; inner: k, omega)
//     contracted with the adjoint and the state -- forward-over-reverse.
#pragma once
#include "engine.cuh"
#include "secular.cuh"

#ifdef MD200_HOST_SECULAR
#define MD200_HD __host__ __device__
#else
#define MD200_HD __device__
#endif

namespace md200 {

using D2 = Dual<double, 2>;  // value, d/dk, d/domega
using DD = Dual<D2, 2>;      // second order in (k, omega)
using P4 = Dual<D2, 4>;      // d/d(h, vp, vs, rho) of one row, of (k, omega) duals

constexpr int JAC_SEG = 12;     // layer steps per recomputed segment
constexpr int JAC_MAXSEG = 12;  // checkpoints: up to 144 layer steps (145 rows)
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
  P4 h, ivp, ivs, vs2, rho, irho, mu, imu;
};
MD200_FN RowP4 row_p4(const double *tab, int Ls, int j) {
  const double h = tab[j], ivp = tab[Ls + j], ivs = tab[2 * Ls + j], vs2 = tab[3 * Ls + j];
  const double rho = tab[4 * Ls + j], irho = tab[5 * Ls + j], imu = tab[6 * Ls + j], vs = tab[8 * Ls + j];
  RowP4 r;
  r.h = seed4(h, 0, 1.);
  r.ivp = seed4(ivp, 1, -ivp * ivp);
  r.ivs = vs > 0. ? seed4(ivs, 2, -ivs * ivs) : P4(0.);
  r.vs2 = seed4(vs2, 2, 2. * vs);
  r.rho = seed4(rho, 3, 1.);
  r.irho = seed4(irho, 3, -irho * irho);
  r.mu = r.rho * r.vs2;
  r.imu = P4(imu);
  if (vs > 0.) {
    r.imu.d[2] = D2(-2. * imu / vs);
    r.imu.d[3] = D2(-imu / rho);
  }
  return r;
}

// e <- M^T lam for the matrix of RayleighEntries (value parts of P4 entries).
MD200_FN void rayleigh_apply_transpose(const RayleighEntries<P4> &X, const D2 &k2, D2 lam[5]) {
  const D2 t = k2 * -2.;
  const D2 l0 = lam[0], l1 = lam[1], l2 = lam[2], l3 = lam[3], l4 = lam[4];
  lam[0] = X.A.v * l0 + X.D.v * l1 + X.I.v * l2 + X.C.v * l3 + X.Lm.v * l4;
  lam[1] = X.E.v * l0 + X.B.v * l1 + X.G.v * l2 + X.M.v * l3 + X.C.v * l4;
  lam[2] = t * (X.J.v * l0 + X.H.v * l1 + X.G.v * l3 + X.I.v * l4) + X.K.v * l2;
  lam[3] = X.F.v * l0 + X.Nn.v * l1 + X.H.v * l2 + X.B.v * l3 + X.D.v * l4;
  lam[4] = X.O.v * l0 + X.F.v * l1 + X.J.v * l2 + X.E.v * l3 + X.A.v * l4;
}

// Derivatives of (F, F_k, F_w) along one row's parameters, as D2 numbers
// (value: F_m; d[0]: F_km; d[1]: F_wm).
struct RowGrad {
  D2 g[4];
};

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
  const double k0 = w / c;
  // (k, omega) duals and their second-order lifts
  D2 k, wd;
  k.v = k0; k.d[0] = 1.; k.d[1] = 0.;
  wd.v = w; wd.d[0] = 0.; wd.d[1] = 1.;
  const D2 iw = D2(1) / wd, iw2 = iw * iw, k2 = k * k;
  DD kk, ww;
  kk.v = k; kk.d[0] = D2(1); kk.d[1] = D2(0);
  ww.v = wd; ww.d[0] = D2(0); ww.d[1] = D2(1);
  const DD iwx = DD(1) / ww, iw2x = iwx * iwx, k2x = kk * kk;

  D2 ck[JAC_MAXSEG][5];
  int ex[JAC_MAX_STEPS];
  int ex0 = 0, pex = 0;
  constexpr int NV = WAVE ? 2 : 5;

  // ---- 1. forward sweep (second order), exponents and checkpoints ----
  DD e[NV];
  if constexpr (WAVE == 0) {
    rayleigh_start<DD, double>(e, kk, k2x, ww, iw2x, m.ivp(last), m.ivs(last), m.vs2(last), m.rho(last));
  } else {
    const DD kb = ww * m.ivs(last);
    DD r, ir;
    radical(kk, kb, &r, &ir);
    e[0] = r * m.rho(last);
    e[1] = DD(1) * (m.ivs(last) * m.ivs(last));
  }
  if constexpr (WAVE == 0) ex0 = scale_vector(e, 5, tiny);
  for (int s = 0; s < nsteps; ++s) {
    const int l = last - 1 - s;
    if (s % JAC_SEG == 0)
      for (int i = 0; i < NV; ++i) ck[s / JAC_SEG][i] = e[i].v;
    if constexpr (WAVE == 0) {
      rayleigh_layer<DD, double>(e, kk, k2x, ww, iw2x, m.h(l), m.ivp(l), m.vs2(l), m.ivs(l), m.rho(l), m.irho(l));
    } else {
      const DD kj = ww * m.ivs(l);
      DD r, ir, cq, y, z;
      radical(kk, kj, &r, &ir);
      love_entries<DD, double>(kk, kj, r, ir, m.h(l), &cq, &y, &z);
      const double mu = m.rho(l) * m.vs2(l);
      const DD u = e[0] * cq + e[1] * z * mu;
      const DD v = e[0] * y * m.imu(l) + e[1] * cq;
      e[0] = u;
      e[1] = v;
    }
    ex[s] = scale_vector(e, NV, tiny);
  }
  // top: the secular value as a function of the final state
  DD F;
  DD cpx, wvx;
  if (WAVE == 0 && top) {
    water_top<DD, double>(kk, ww, m.h(0), m.ivp(0), &cpx, &wvx);
    DD pair[2] = {cpx * e[0], wvx * e[1] * m.rho(0)};
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
  const P4 kP = lift4(k), k2P = lift4(k2), wP = lift4(wd), iw2P = lift4(iw2);
  D2 lam[NV];
  for (int i = 0; i < NV; ++i) lam[i] = D2(0);
  if (WAVE == 0 && top) {
    // F = (cp e0 - wv e1 rho0) 2^-pex, with the fluid row's own parameters
    const double rp = pow2(-pex);
    // final state (value parts of the forward sweep)
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
      if constexpr (WAVE == 0) {
        rayleigh_layer<D2, double>(x, k, k2, wd, iw2, m.h(l), m.ivp(l), m.vs2(l), m.ivs(l), m.rho(l), m.irho(l));
      } else {
        const D2 kj = wd * m.ivs(l);
        D2 r, ir, cq, y, z;
        radical(k, kj, &r, &ir);
        love_entries<D2, double>(k, kj, r, ir, m.h(l), &cq, &y, &z);
        const double mu = m.rho(l) * m.vs2(l);
        const D2 u = x[0] * cq + x[1] * z * mu;
        const D2 v = x[0] * y * m.imu(l) + x[1] * cq;
        x[0] = u;
        x[1] = v;
      }
      const double r = pow2(-ex[s]);
      for (int i = 0; i < NV; ++i) x[i] = x[i] * r;
    }
    // reverse through the segment, top layer first
    for (int s = s1 - 1; s >= s0; --s) {
      const int l = last - 1 - s;
      const double r = pow2(-ex[s]);
      const RowP4 row = row_p4(tab, Ls, l);
      RowGrad g;
      if constexpr (WAVE == 0) {
        RayleighEntries<P4> X;
        rayleigh_entries<P4, P4>(X, kP, k2P, wP, iw2P, row.h, row.ivp, row.vs2, row.ivs, row.rho, row.irho);
        P4 y[5];
        for (int i = 0; i < 5; ++i) y[i] = lift4(st[s - s0][i]);
        rayleigh_apply<P4>(X, k2P, y);
        for (int p = 0; p < 4; ++p) {
          D2 acc = lam[0] * y[0].d[p];
          for (int i = 1; i < 5; ++i) acc = acc + lam[i] * y[i].d[p];
          g.g[p] = acc * r;
        }
        rayleigh_apply_transpose(X, k2, lam);
        for (int i = 0; i < 5; ++i) lam[i] = lam[i] * r;
      } else {
        const P4 kj = wP * row.ivs;
        P4 rr, ir, cq, y, z;
        radical(kP, kj, &rr, &ir);
        love_entries<P4, P4>(kP, kj, rr, ir, row.h, &cq, &y, &z);
        const P4 e0 = lift4(st[s - s0][0]), e1 = lift4(st[s - s0][1]);
        const P4 u = e0 * cq + e1 * z * row.mu;
        const P4 v = e0 * y * row.imu + e1 * cq;
        for (int p = 0; p < 4; ++p) g.g[p] = (lam[0] * u.d[p] + lam[1] * v.d[p]) * r;
        const D2 l0 = lam[0], l1 = lam[1];
        lam[0] = (l0 * cq.v + l1 * (y.v * row.imu.v)) * r;
        lam[1] = (l0 * (z.v * row.mu.v) + l1 * cq.v) * r;
      }
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
