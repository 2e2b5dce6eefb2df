/*
 * md_oracle.c -- CPU restatement of modisp's FP64 dispersion numerics.
 *
 * TEST INFRASTRUCTURE ONLY (the oracle).  The test suite, smoke() and
 * bench.py's CPU-baseline leg load it as the checker; the product never does.
 *
 * The double-precision routines restate the reference arithmetic in the same
 * operation order so that, compiled with -ffp-contract=off against the same
 * libm, they reproduce the reference CPU engine's secular values bit for bit
 * (pinned in tests/test_oracle.py).  The long-double complex-step routines are
 * an independent derivative check used for group velocities and Jacobians; the
 * reference estimates group velocity by finite differences instead
 * (cpp/common/group_velocity.hpp:205-283).
 */
#include "md_oracle.h"

#include <complex.h>
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define MDO_TWO_PI 6.283185307179586476925286766559

typedef long double complex cld;

/* ------------------------------------------------------------------------- */
/* Rayleigh: normalized Dunkin compound-matrix recurrence                     */
/* cpp/common/dunkin.hpp:82-159 (dunkin_var), :171-221 (dunkin_dnka),        */
/* :335-348 (max amplitude), :358-448 (dunkin_secular, NORMALIZE = true).    */
/* ------------------------------------------------------------------------- */

/* Eigenfunction products of one layer (dunkin.hpp:82-159, FAST = false). */
static void layer_products(double p, double q, double ra, double rb, double wvno,
                           double xka, double xkb, double dpth, double out[10]) {
  double cosp = 0., w = 0., x = 0., cosq = 0., y = 0., z = 0., pex = 0., sex = 0.;
  if (wvno < xka) {
    const double sp = sin(p), cp = cos(p);
    w = sp / ra;
    x = -ra * sp;
    cosp = cp;
  } else if (wvno == xka) {
    cosp = 1.;
    w = dpth;
    x = 0.;
  } else {
    pex = p;
    const double fac = (p < 16.) ? exp(-2. * p) : 0.;
    cosp = (1. + fac) * 0.5;
    const double sp = (1. - fac) * 0.5;
    w = sp / ra;
    x = ra * sp;
  }
  if (wvno < xkb) {
    const double sq = sin(q), cq = cos(q);
    y = sq / rb;
    z = -rb * sq;
    cosq = cq;
  } else if (wvno == xkb) {
    cosq = 1.;
    y = dpth;
    z = 0.;
  } else {
    sex = q;
    const double fac = (q < 16.) ? exp(-2. * q) : 0.;
    cosq = (1. + fac) * 0.5;
    const double sq = (1. - fac) * 0.5;
    y = sq / rb;
    z = rb * sq;
  }
  const double exa = pex + sex;
  out[0] = (exa == 0.) ? 1. : ((exa < 60.) ? exp(-exa) : 0.); /* a0 */
  out[1] = cosp * cosq;                                         /* cpcq */
  out[2] = cosp * y;                                            /* cpy */
  out[3] = cosp * z;                                            /* cpz */
  out[4] = cosq * w;                                            /* cqw */
  out[5] = cosq * x;                                            /* cqx */
  out[6] = x * y;                                               /* xy */
  out[7] = x * z;                                               /* xz */
  out[8] = w * y;                                               /* wy */
  out[9] = w * z;                                               /* wz */
}

/* The 5x5 compound layer matrix (dunkin.hpp:171-221). */
static void layer_matrix(double wvno2, double gam, double gammk, double rho,
                         const double v[10], double ca[5][5]) {
  const double a0 = v[0], cpcq = v[1], cpy = v[2], cpz = v[3], cqw = v[4], cqx = v[5];
  const double xy = v[6], xz = v[7], wy = v[8], wz = v[9];
  const double gamm1 = gam - 1.;
  const double twgm1 = gam + gamm1;
  const double gmgmk = gam * gammk;
  const double gmgm1 = gam * gamm1;
  const double gm1sq = gamm1 * gamm1;
  const double rho2 = rho * rho;
  const double a0pq = a0 - cpcq;
  const double t = -2. * wvno2;

  ca[0][0] = cpcq - 2. * gmgm1 * a0pq - gmgmk * xz - wvno2 * gm1sq * wy;
  ca[0][1] = (wvno2 * cpy - cqx) / rho;
  ca[0][2] = -(twgm1 * a0pq + gammk * xz + wvno2 * gamm1 * wy) / rho;
  ca[0][3] = (cpz - wvno2 * cqw) / rho;
  ca[0][4] = -(2. * wvno2 * a0pq + xz + wvno2 * wvno2 * wy) / rho2;

  ca[1][0] = (gmgmk * cpz - gm1sq * cqw) * rho;
  ca[1][1] = cpcq;
  ca[1][2] = gammk * cpz - gamm1 * cqw;
  ca[1][3] = -wz;
  ca[1][4] = ca[0][3];

  ca[3][0] = (gm1sq * cpy - gmgmk * cqx) * rho;
  ca[3][1] = -xy;
  ca[3][2] = gamm1 * cpy - gammk * cqx;
  ca[3][3] = ca[1][1];
  ca[3][4] = ca[0][1];

  ca[4][0] = -(2. * gmgmk * gm1sq * a0pq + gmgmk * gmgmk * xz + gm1sq * gm1sq * wy) * rho2;
  ca[4][1] = ca[3][0];
  ca[4][2] = -(gammk * gamm1 * twgm1 * a0pq + gam * gammk * gammk * xz + gamm1 * gm1sq * wy) * rho;
  ca[4][3] = ca[1][0];
  ca[4][4] = ca[0][0];

  ca[2][0] = t * ca[4][2];
  ca[2][1] = t * ca[3][2];
  ca[2][2] = a0 + 2. * (cpcq - ca[0][0]);
  ca[2][3] = t * ca[1][2];
  ca[2][4] = t * ca[0][2];
}

double mdo_rayleigh(const double *d, const double *a, const double *b, const double *rho,
                    int L, double omega, double c, double *shape) {
  const double wvno = omega / c;
  const double wvno2 = wvno * wvno;
  const int last = L - 1;
  const int water = b[0] == 0. ? 1 : 0;

  const double xka0 = omega / a[last];
  const double xkb0 = omega / b[last];
  double ra = sqrt((wvno + xka0) * fabs(wvno - xka0));
  double rb = sqrt((wvno + xkb0) * fabs(wvno - xkb0));
  double t = b[last] / omega;
  double gammk = 2. * t * t;
  double gam = gammk * wvno2;
  const double gamm1 = gam - 1.;
  const double rho_hs = rho[last];

  double e[5];
  e[0] = rho_hs * rho_hs * (gamm1 * gamm1 - gam * gammk * ra * rb);
  e[1] = -rho_hs * ra;
  e[2] = rho_hs * (gamm1 - gammk * ra * rb);
  e[3] = rho_hs * rb;
  e[4] = wvno2 - ra * rb;

  for (int m = L - 2; m >= water; --m) {
    const double xka = omega / a[m];
    const double xkb = omega / b[m];
    t = b[m] / omega;
    gammk = 2. * t * t;
    gam = gammk * wvno2;
    ra = sqrt((wvno + xka) * fabs(wvno - xka));
    rb = sqrt((wvno + xkb) * fabs(wvno - xkb));
    const double dpth = d[m];
    double v[10], ca[5][5], ee[5];
    layer_products(ra * dpth, rb * dpth, ra, rb, wvno, xka, xkb, dpth, v);
    layer_matrix(wvno2, gam, gammk, rho[m], v, ca);
    for (int i = 0; i < 5; ++i) {
      double s = 0.;
      for (int j = 0; j < 5; ++j) s += e[j] * ca[j][i];
      ee[i] = s;
    }
    double scale = 0.;
    for (int i = 0; i < 5; ++i) {
      const double mag = fabs(ee[i]);
      if (mag > scale) scale = mag;
    }
    if (scale < 1.0e-40) scale = 1.;
    for (int i = 0; i < 5; ++i) e[i] = ee[i] / scale;
  }

  if (water) { /* dunkin.hpp:427-442 */
    const double ka = omega / a[0];
    const double rf = sqrt((wvno + ka) * fabs(wvno - ka));
    const double p = rf * d[0];
    double cp, w;
    if (wvno < ka) {
      const double sn = sin(p);
      cp = cos(p);
      w = sn / rf;
    } else if (wvno == ka) {
      cp = 1.;
      w = d[0];
    } else {
      const double zz = (p < 16.) ? exp(-2. * p) : 0.;
      cp = (1. + zz) * .5;
      w = (1. - zz) * .5 / rf;
    }
    const double t0 = cp * e[0], t1 = rho[0] * w * e[1];
    const double scale = fmax(1., fmax(fabs(t0), fabs(t1)));
    if (shape) {
      const double u = t0 / scale, vv = t1 / scale;
      *shape = (u - vv) / sqrt(u * u + vv * vv + 1e-300);
    }
    return t0 / scale - t1 / scale;
  }
  if (shape) {
    double other = 1e-300;
    for (int i = 1; i < 5; ++i) other += e[i] * e[i];
    *shape = e[0] / sqrt(e[0] * e[0] + other);
  }
  return e[0];
}

/* ------------------------------------------------------------------------- */
/* Love: SH 2-vector recurrence (cpp/common/physics.hpp:33-53)               */
/* ------------------------------------------------------------------------- */
double mdo_love(const double *h, const double *vs, const double *rho, int L, double omega,
                double c, double *shape) {
  const int top = vs[0] == 0. ? 1 : 0, last = L - 1;
  const double k = omega / c, kb = omega / vs[last];
  double e1 = rho[last] * sqrt((k + kb) * fabs(k - kb));
  double e2 = 1. / (vs[last] * vs[last]);
  for (int j = last - 1; j >= top; --j) {
    const double mu = rho[j] * vs[j] * vs[j], ka = omega / vs[j];
    const double r = sqrt((k + ka) * fabs(k - ka)), q = r * h[j];
    double cq, y, z;
    if (k < ka) {
      const double sn = sin(q);
      cq = cos(q);
      y = sn / r;
      z = -r * sn;
    } else if (k == ka) {
      cq = 1.;
      y = h[j];
      z = 0.;
    } else {
      const double f = q < 16. ? exp(-2. * q) : 0.;
      cq = (1. + f) * .5;
      y = (1. - f) * .5 / r;
      z = (1. - f) * .5 * r;
    }
    const double u = e1 * cq + e2 * mu * z, v = e1 * y / mu + e2 * cq;
    double s = fmax(fabs(u), fabs(v));
    if (s < 1e-40) s = 1.;
    e1 = u / s;
    e2 = v / s;
  }
  if (shape) *shape = e1 / sqrt(e1 * e1 + e2 * e2 + 1e-300);
  return e1;
}

double mdo_secular(const double *h, const double *vp, const double *vs, const double *rho,
                   int L, int wave, double omega, double c, double *shape) {
  return wave ? mdo_love(h, vs, rho, L, omega, c, shape)
              : mdo_rayleigh(h, vp, vs, rho, L, omega, c, shape);
}

/* ------------------------------------------------------------------------- */
/* Unwrapped SH phase (cpp/common/love_phase.hpp:246-277)                    */
/* ------------------------------------------------------------------------- */
static int finite_value(double x) { return x == x && fabs(x) != INFINITY; }

static double unwrap(double raw, double previous) {
  return previous + atan2(sin(raw - previous), cos(raw - previous));
}

double mdo_love_phase(const double *h, const double *vs, const double *rho, int L,
                      double omega, double c) {
  const int last = L - 1, top = vs[0] == 0. ? 1 : 0;
  const double k = omega / c, khalf = omega / vs[last];
  if (!(k > khalf)) return NAN;
  double scale = rho[last] * vs[last] * vs[last] * sqrt((k + khalf) * (k - khalf));
  double theta = MDO_TWO_PI * .125;
  for (int j = last - 1; j >= top; --j) {
    if (h[j] == 0.) continue;
    const double mu = rho[j] * vs[j] * vs[j], kb = omega / vs[j];
    const double r = sqrt(fabs((k + kb) * (k - kb))), next = mu * (r > 0. ? r : 1. / h[j]);
    if (!(scale > 0.) || !(next > 0.) || !finite_value(scale / next)) return NAN;
    theta = unwrap(atan2((scale / next) * sin(theta), cos(theta)), theta);
    scale = next;
    if (k < kb) {
      theta -= r * h[j];
    } else {
      const double x = sin(theta), y = cos(theta);
      double u, t;
      if (r == 0.) {
        t = x;
        u = y + x * h[j] * scale / mu;
      } else {
        const double e = exp(-2. * r * h[j]), cq = .5 * (1. + e), sn = .5 * (1. - e);
        t = x * cq + y * sn;
        u = y * cq + x * sn;
      }
      if (fmax(fabs(t), fabs(u)) < 1e-14) return NAN;
      theta = unwrap(atan2(t, u), theta);
    }
    if (!finite_value(theta) || fabs(theta) > 1048576.) return NAN;
  }
  return theta;
}

/* ------------------------------------------------------------------------- */
/* Search window (cpp/common/physics.hpp:140-175, cpp/cpu/solver.cpp:781-790) */
/* ------------------------------------------------------------------------- */
static double rayleigh_speed(double vp, double vs) {
  const double ratio = (vs / vp) * (vs / vp);
  double l = 0., h = 1.;
  for (int j = 0; j < 56; ++j) {
    const double x = (l + h) * .5;
    const double f = ((x - 8.) * x + 24. - 16. * ratio) * x - 16. * (1. - ratio);
    if (f < 0.) l = x; else h = x;
  }
  return vs * sqrt((l + h) * .5);
}

static double scholte_speed(double vf, double rf, double vp, double vs, double rs) {
  const double ratio = (vs / vp) * (vs / vp), qf = (vs / vf) * (vs / vf);
  double l = 0., h = fmax(0., fmin(1., vf / vs) * (1. - 1e-12));
  for (int j = 0; j < 64; ++j) {
    const double x = (l + h) * .5, x2 = x * x;
    const double A = sqrt(fmax(0., 1. - ratio * x2)), B = sqrt(fmax(0., 1. - x2));
    const double f = 4. * (1. + ratio - ratio * x2) / (1. + A * B) - 4. + x2 +
                     (rf / rs) * x2 * A / sqrt(fmax(1e-30, 1. - qf * x2));
    if (f < 0.) l = x; else h = x;
  }
  return vs * (l + h) * .5;
}

void mdo_bounds(const double *h, const double *vp, const double *vs, const double *rho,
                int L, int wave, double *lo, double *hi) {
  double seed = 1e300;
  const int top = vs[0] == 0. ? 1 : 0;
  for (int j = top; j < L; ++j) {
    if (h[j] == 0. && j < L - 1) continue;
    const double s = vs[j], p = vp[j];
    if (!wave && !top && s > 0. && .68 * s > seed) {
      const double ratio = s / p;
      if (ratio > 0. && ratio * ratio <= .75) continue;
    }
    double x = wave ? s : rayleigh_speed(p, s);
    if (!wave && top) x = fmin(x, scholte_speed(vp[0], rho[0], p, s, rho[j]));
    seed = fmin(seed, x);
  }
  *lo = .125 * seed;
  *hi = fmin(vs[L - 1], nextafter(vs[L - 1], 0.));
}

/* ------------------------------------------------------------------------- */
/* Brent refinement (cpp/common/refinement.hpp:339-343, :374-396)            */
/* ------------------------------------------------------------------------- */
double mdo_refine(const double *hh, const double *vp, const double *vs, const double *rho,
                  int L, int wave, double w, double a, double b, double fa, double fb,
                  double tol, int *evaluations) {
  int ev = 0;
  if (a == b) return fa == 0. ? a : NAN;
  if (!finite_value(fa) || !finite_value(fb) || ((fa < 0.) == (fb < 0.) && fa != 0. && fb != 0.))
    return NAN;
  if (fa == 0.) return a;
  if (fb == 0.) return b;
  const double big = fmax(fabs(a), fabs(b));
  const double stop = fmax(16. * DBL_EPSILON * big, fmin((b - a) / 64., .125 * tol * big));
  double c = b, fc = fb, d = b - a, e = d;
  double result = NAN;
  for (int j = 0; j < 160; ++j) {
    if ((fb < 0.) == (fc < 0.)) {
      c = a;
      fc = fa;
      e = d = b - a;
    }
    if (fabs(fc) < fabs(fb)) {
      a = b; fa = fb;
      b = c; fb = fc;
      c = a; fc = fa;
    }
    if (fb == 0.) { result = b; break; }
    const double mid = .5 * (c - b), step = .5 * stop;
    if (fabs(c - b) <= stop) { result = .5 * (b + c); break; }
    if (fabs(e) >= step && fabs(fa) > fabs(fb)) {
      const double s = fb / fa;
      double p, q;
      if (a == c) {
        p = 2. * mid * s;
        q = 1. - s;
      } else {
        q = fa / fc;
        const double r = fb / fc;
        p = s * (2. * mid * q * (q - r) - (b - a) * (r - 1.));
        q = (q - 1.) * (r - 1.) * (s - 1.);
      }
      if (p > 0.) q = -q; else p = -p;
      const double old = e;
      e = d;
      if (finite_value(p / q) && 2. * p < fmin(3. * mid * q - fabs(step * q), fabs(old * q))) d = p / q;
      else { d = mid; e = mid; }
    } else {
      d = mid;
      e = mid;
    }
    a = b;
    fa = fb;
    b += fabs(d) > step ? d : (mid > 0. ? step : -step);
    fb = mdo_secular(hh, vp, vs, rho, L, wave, w, b, 0);
    ++ev;
    if (!finite_value(fb)) break;
  }
  if (evaluations) *evaluations += ev;
  return result;
}

/* ------------------------------------------------------------------------- */
/* Dense uniform search (cpp/cpu/solver.cpp:221-252, :329-370;               */
/* cpp/common/physics.hpp:130-138 density, :195-204 workload)                */
/* ------------------------------------------------------------------------- */
static double density(const double *h, const double *vp, const double *vs, int L, int wave,
                      double c) {
  const double ic = 1.0 / (c * c);
  double n = 0.;
  for (int j = 0; j < L - 1; ++j) {
    if (h[j] == 0.) continue;
    const double ivs = vs[j] == 0. ? 0. : 1. / (vs[j] * vs[j]);
    const double ivp = 1. / (vp[j] * vp[j]);
    if (ivs > ic) n += h[j] * sqrt(ivs - ic);
    if (wave == 0 && ivp > ic) n += h[j] * sqrt(ivp - ic);
  }
  return 2. * n;
}

int mdo_dense_roots(const double *h, const double *vp, const double *vs, const double *rho,
                    int L, int wave, double period, double lo, double hi, int K, double tol,
                    double *roots) {
  double need = 32. * density(h, vp, vs, L, wave, hi) / period;
  if (!wave && vs[0] == 0.) {
    const double optical = 2. * h[0] / (period * vp[0]);
    need = fmax(need, 2. * fmax(0., hi - lo) * optical * optical / vp[0]);
  }
  if (!finite_value(need) || need > 524288.) return -1;
  long cells = 32768;
  while (cells < need) cells *= 2;
  const double omega = MDO_TWO_PI / period;
  int n = 0;
  double x0 = lo, f0 = mdo_secular(h, vp, vs, rho, L, wave, omega, lo, 0);
  double fprev = NAN; /* value before x0, for exact-zero sign tests */
  for (long j = 1; j <= cells && n < K; ++j) {
    const double x1 = lo + (hi - lo) * j / cells;
    const double f1 = mdo_secular(h, vp, vs, rho, L, wave, omega, x1, 0);
    if (!finite_value(f0) || !finite_value(f1)) return -1;
    if (f0 == 0.) {
      if (f1 == 0. || fprev == 0.) return -1;
      if ((j > 1 && signbit(fprev) != signbit(f1)) || j == 1) roots[n++] = x0;
      else return -1;
    } else if (f1 != 0. && signbit(f0) != signbit(f1)) {
      const double r = mdo_refine(h, vp, vs, rho, L, wave, omega, x0, x1, f0, f1, tol, 0);
      if (!finite_value(r)) return -1;
      roots[n++] = r;
    }
    if (j == cells && f1 == 0. && n < K) {
      if (f0 == 0.) return -1;
      roots[n++] = x1;
    }
    fprev = f0;
    x0 = x1;
    f0 = f1;
  }
  return n;
}

/* ------------------------------------------------------------------------- */
/* Complex-step derivatives in long double                                   */
/* The same recurrences as above with every input complex; branch choices    */
/* and normalisation scales use real parts only, so the imaginary part of    */
/* the result is the derivative of the unnormalised function times the same  */
/* positive scale as the real part.  Ratios of derivatives at a root are     */
/* therefore exact.                                                          */
/* ------------------------------------------------------------------------- */
static cld cx_root_term(cld k, cld kb) { /* (k + kb) * |k - kb| with a real-part sign */
  return creall(k) >= creall(kb) ? (k + kb) * (k - kb) : (k + kb) * (kb - k);
}

/* Near k = kv the wave blocks are taken as power series in y = (k^2 - kv^2) h^2,
 * unscaled and without the square root: cs = C(y), sr = h S(y),
 * rs = (k^2 - kv^2) h S(y), C = sum y^n / (2n)!, S = sum y^n / (2n+1)!
 * (cos / sin for y < 0, cosh / sinh for y > 0).  The direct form's complex-step
 * derivative of sin(r h) / r cancels to a relative error of about
 * eps / (r h)^2; the series has no such cancellation.  Terms up to y^8 leave
 * < 1e-28 relative truncation error for |y| < 1e-2. */
static int cx_series(cld k, cld kv, cld h, cld *cs, cld *sr, cld *rs) {
  const cld D = (k + kv) * (k - kv), y = D * h * h;
  if (!(fabsl(creall(y)) < 1e-2L)) return 0;
  long double inv_fact[18];
  inv_fact[0] = 1.L;
  for (int n = 1; n < 18; ++n) inv_fact[n] = inv_fact[n - 1] / (long double)n;
  cld C = 0.L, S = 0.L;
  for (int n = 8; n >= 0; --n) {
    C = C * y + inv_fact[2 * n];
    S = S * y + inv_fact[2 * n + 1];
  }
  *cs = C;
  *sr = S * h;
  *rs = D * S * h;
  return 1;
}

static cld cx_rayleigh(const cld *d, const cld *a, const cld *b, const cld *rho, int L,
                       cld wvno, cld omega) {
  const cld wvno2 = wvno * wvno;
  const int last = L - 1;
  const int water = creall(b[0]) == 0.L ? 1 : 0;
  cld xka = omega / a[last], xkb = omega / b[last];
  cld ra = csqrtl(cx_root_term(wvno, xka)), rb = csqrtl(cx_root_term(wvno, xkb));
  cld t = b[last] / omega, gammk = 2.L * t * t, gam = gammk * wvno2, gamm1 = gam - 1.L;
  const cld rh = rho[last];
  cld e[5];
  e[0] = rh * rh * (gamm1 * gamm1 - gam * gammk * ra * rb);
  e[1] = -rh * ra;
  e[2] = rh * (gamm1 - gammk * ra * rb);
  e[3] = rh * rb;
  e[4] = wvno2 - ra * rb;
  for (int m = L - 2; m >= water; --m) {
    xka = omega / a[m];
    xkb = omega / b[m];
    t = b[m] / omega;
    gammk = 2.L * t * t;
    gam = gammk * wvno2;
    ra = csqrtl(cx_root_term(wvno, xka));
    rb = csqrtl(cx_root_term(wvno, xkb));
    const cld dp = d[m], p = ra * dp, q = rb * dp;
    cld cosp, w, x, cosq, y, z, pex = 0.L, sex = 0.L;
    if (cx_series(wvno, xka, dp, &cosp, &w, &x)) {
    } else if (creall(wvno) < creall(xka)) {
      const cld sp = csinl(p);
      cosp = ccosl(p);
      w = sp / ra;
      x = -ra * sp;
    } else if (creall(wvno) == creall(xka)) {
      cosp = 1.L; w = dp; x = 0.L;
    } else {
      pex = p;
      const cld fac = creall(p) < 16.L ? cexpl(-2.L * p) : 0.L;
      cosp = (1.L + fac) * .5L;
      const cld sp = (1.L - fac) * .5L;
      w = sp / ra;
      x = ra * sp;
    }
    if (cx_series(wvno, xkb, dp, &cosq, &y, &z)) {
    } else if (creall(wvno) < creall(xkb)) {
      const cld sq = csinl(q);
      cosq = ccosl(q);
      y = sq / rb;
      z = -rb * sq;
    } else if (creall(wvno) == creall(xkb)) {
      cosq = 1.L; y = dp; z = 0.L;
    } else {
      sex = q;
      const cld fac = creall(q) < 16.L ? cexpl(-2.L * q) : 0.L;
      cosq = (1.L + fac) * .5L;
      const cld sq = (1.L - fac) * .5L;
      y = sq / rb;
      z = rb * sq;
    }
    const cld exa = pex + sex;
    const cld a0 = creall(exa) == 0.L && cimagl(exa) == 0.L ? 1.L
                   : (creall(exa) < 60.L ? cexpl(-exa) : 0.L);
    const cld cpcq = cosp * cosq, cpy = cosp * y, cpz = cosp * z, cqw = cosq * w, cqx = cosq * x;
    const cld xy = x * y, xz = x * z, wy = w * y, wz = w * z;
    const cld rl = rho[m], rho2 = rl * rl;
    const cld gm1 = gam - 1.L, twgm1 = gam + gm1, gmgmk = gam * gammk, gmgm1 = gam * gm1,
              gm1sq = gm1 * gm1, a0pq = a0 - cpcq, tt = -2.L * wvno2;
    cld ca[5][5];
    ca[0][0] = cpcq - 2.L * gmgm1 * a0pq - gmgmk * xz - wvno2 * gm1sq * wy;
    ca[0][1] = (wvno2 * cpy - cqx) / rl;
    ca[0][2] = -(twgm1 * a0pq + gammk * xz + wvno2 * gm1 * wy) / rl;
    ca[0][3] = (cpz - wvno2 * cqw) / rl;
    ca[0][4] = -(2.L * wvno2 * a0pq + xz + wvno2 * wvno2 * wy) / rho2;
    ca[1][0] = (gmgmk * cpz - gm1sq * cqw) * rl;
    ca[1][1] = cpcq;
    ca[1][2] = gammk * cpz - gm1 * cqw;
    ca[1][3] = -wz;
    ca[1][4] = ca[0][3];
    ca[3][0] = (gm1sq * cpy - gmgmk * cqx) * rl;
    ca[3][1] = -xy;
    ca[3][2] = gm1 * cpy - gammk * cqx;
    ca[3][3] = ca[1][1];
    ca[3][4] = ca[0][1];
    ca[4][0] = -(2.L * gmgmk * gm1sq * a0pq + gmgmk * gmgmk * xz + gm1sq * gm1sq * wy) * rho2;
    ca[4][1] = ca[3][0];
    ca[4][2] = -(gammk * gm1 * twgm1 * a0pq + gam * gammk * gammk * xz + gm1 * gm1sq * wy) * rl;
    ca[4][3] = ca[1][0];
    ca[4][4] = ca[0][0];
    ca[2][0] = tt * ca[4][2];
    ca[2][1] = tt * ca[3][2];
    ca[2][2] = a0 + 2.L * (cpcq - ca[0][0]);
    ca[2][3] = tt * ca[1][2];
    ca[2][4] = tt * ca[0][2];
    cld ee[5];
    long double scale = 0.L;
    for (int i = 0; i < 5; ++i) {
      cld s = 0.L;
      for (int j = 0; j < 5; ++j) s += e[j] * ca[j][i];
      ee[i] = s;
      if (fabsl(creall(s)) > scale) scale = fabsl(creall(s));
    }
    if (scale < 1e-40L) scale = 1.L;
    for (int i = 0; i < 5; ++i) e[i] = ee[i] / scale;
  }
  if (water) {
    const cld ka = omega / a[0];
    const cld rf = csqrtl(cx_root_term(wvno, ka));
    const cld p = rf * d[0];
    cld cp, w, unused;
    if (cx_series(wvno, ka, d[0], &cp, &w, &unused)) {
    } else if (creall(wvno) < creall(ka)) {
      cp = ccosl(p);
      w = csinl(p) / rf;
    } else if (creall(wvno) == creall(ka)) {
      cp = 1.L; w = d[0];
    } else {
      const cld zz = creall(p) < 16.L ? cexpl(-2.L * p) : 0.L;
      cp = (1.L + zz) * .5L;
      w = (1.L - zz) * .5L / rf;
    }
    const cld t0 = cp * e[0], t1 = rho[0] * w * e[1];
    const long double scale = fmaxl(1.L, fmaxl(fabsl(creall(t0)), fabsl(creall(t1))));
    return (t0 - t1) / scale;
  }
  return e[0];
}

static cld cx_love(const cld *h, const cld *vs, const cld *rho, int L, cld omega, cld k) {
  const int top = creall(vs[0]) == 0.L ? 1 : 0, last = L - 1;
  const cld kb = omega / vs[last];
  cld e1 = rho[last] * csqrtl(cx_root_term(k, kb));
  cld e2 = 1.L / (vs[last] * vs[last]);
  for (int j = last - 1; j >= top; --j) {
    const cld mu = rho[j] * vs[j] * vs[j], ka = omega / vs[j];
    const cld r = csqrtl(cx_root_term(k, ka)), q = r * h[j];
    cld cq, y, z;
    if (cx_series(k, ka, h[j], &cq, &y, &z)) {
    } else if (creall(k) < creall(ka)) {
      const cld sn = csinl(q);
      cq = ccosl(q);
      y = sn / r;
      z = -r * sn;
    } else if (creall(k) == creall(ka)) {
      cq = 1.L; y = h[j]; z = 0.L;
    } else {
      const cld f = creall(q) < 16.L ? cexpl(-2.L * q) : 0.L;
      cq = (1.L + f) * .5L;
      y = (1.L - f) * .5L / r;
      z = (1.L - f) * .5L * r;
    }
    const cld u = e1 * cq + e2 * mu * z, v = e1 * y / mu + e2 * cq;
    long double s = fmaxl(fabsl(creall(u)), fabsl(creall(v)));
    if (s < 1e-40L) s = 1.L;
    e1 = u / s;
    e2 = v / s;
  }
  return e1;
}

typedef struct {
  cld *h, *vp, *vs, *rho;
  int L, wave;
} CxModel;

static void cx_load(CxModel *m, const double *h, const double *vp, const double *vs,
                    const double *rho, int L, int wave) {
  m->L = L;
  m->wave = wave;
  m->h = (cld *)malloc(sizeof(cld) * 4 * (size_t)L);
  m->vp = m->h + L;
  m->vs = m->vp + L;
  m->rho = m->vs + L;
  for (int j = 0; j < L; ++j) {
    m->h[j] = h[j];
    m->vp[j] = vp[j];
    m->vs[j] = vs[j];
    m->rho[j] = rho[j];
  }
}

static cld cx_eval(const CxModel *m, cld k, cld omega) {
  return m->wave ? cx_love(m->h, m->vs, m->rho, m->L, omega, k)
                 : cx_rayleigh(m->h, m->vp, m->vs, m->rho, m->L, k, omega);
}

static const long double STEP = 1e-40L;

void mdo_derivatives(const double *h, const double *vp, const double *vs, const double *rho,
                     int L, int wave, double omega, double c, double *dfdk, double *dfdw) {
  CxModel m;
  cx_load(&m, h, vp, vs, rho, L, wave);
  const long double w = omega, k = w / (long double)c;
  *dfdk = (double)(cimagl(cx_eval(&m, k + I * STEP, w)) / STEP);
  *dfdw = (double)(cimagl(cx_eval(&m, k, w + I * STEP)) / STEP);
  free(m.h);
}

static long double real_eval(const CxModel *m, long double omega, long double c) {
  return creall(cx_eval(m, omega / c, omega));
}

int mdo_group(const double *h, const double *vp, const double *vs, const double *rho, int L,
              int wave, double omega, double root, double lower, double upper, double *group) {
  CxModel m;
  cx_load(&m, h, vp, vs, rho, L, wave);
  const long double w = omega;
  /* Bracket the root inside (lower, upper) by widening a small window, then bisect in
   * long double to the last bit. */
  long double span = 1e-9L * root, a = 0.L, b = 0.L, fa = 0.L, fb = 0.L;
  int found = 0;
  for (int attempt = 0; attempt < 40 && !found; ++attempt, span *= 2.L) {
    a = fmaxl(root - span, 0.5L * (root + lower));
    b = fminl(root + span, 0.5L * (root + upper));
    fa = real_eval(&m, w, a);
    fb = real_eval(&m, w, b);
    if ((fa < 0.L) != (fb < 0.L) || fa == 0.L || fb == 0.L) found = 1;
  }
  if (!found) { free(m.h); *group = NAN; return 1; }
  for (int j = 0; j < 200 && b - a > 4.L * LDBL_EPSILON * b; ++j) {
    if (fa == 0.L) { b = a; break; }
    if (fb == 0.L) { a = b; break; }
    const long double mid = .5L * (a + b), fm = real_eval(&m, w, mid);
    if ((fm < 0.L) == (fa < 0.L)) { a = mid; fa = fm; } else { b = mid; fb = fm; }
  }
  const long double c = .5L * (a + b), k = w / c;
  const long double fk = cimagl(cx_eval(&m, k + I * STEP, w)) / STEP;
  const long double fw = cimagl(cx_eval(&m, k, w + I * STEP)) / STEP;
  free(m.h);
  *group = (double)(-fk / fw);
  return 0;
}

void mdo_parameter_derivatives(const double *h, const double *vp, const double *vs,
                               const double *rho, int L, int wave, double omega, double c,
                               double *dfdtheta, double *dfdc) {
  CxModel m;
  cx_load(&m, h, vp, vs, rho, L, wave);
  const long double w = omega, k = w / (long double)c;
  cld *blocks[4] = {m.h, m.vp, m.vs, m.rho};
  for (int p = 0; p < 4; ++p) {
    for (int j = 0; j < L; ++j) {
      const cld saved = blocks[p][j];
      blocks[p][j] = saved + I * STEP;
      dfdtheta[p * L + j] = (double)(cimagl(cx_eval(&m, k, w)) / STEP);
      blocks[p][j] = saved;
    }
  }
  /* dF/dc at fixed omega: perturb c through k = omega / c. */
  const cld kc = w / ((long double)c + I * STEP);
  *dfdc = (double)(cimagl(cx_eval(&m, kc, w)) / STEP);
  free(m.h);
}

/* ------------------------------------------------------------------------- */
/* Legacy uniform-grid path, stage 2 (cpp/cuda/refine.cuh:131-317): one mode */
/* at a time, each walking the row from the start as the reference's thread  */
/* for that mode does; FP64 values from mdo_rayleigh (the normalised Dunkin   */
/* recurrence, dunkin_secular_omega<double, true>).                          */
/* ------------------------------------------------------------------------- */
static double uni_c(double cmin, double dc, int i) { return fma(dc, (double)i, cmin); } /* refine.cuh:33-35 */

typedef struct {
  const double *h, *vp, *vs, *rho;
  int L;
  double omega;
} UniModel;

static double uni_f(const UniModel *m, double c) { return mdo_rayleigh(m->h, m->vp, m->vs, m->rho, m->L, m->omega, c, NULL); }

/* refine.cuh:63-80 */
static int uni_retry(const UniModel *m, int cell, int dir, int i_last, double cmin, double dc, double *lo,
                     double *hi, double *flo) {
  const int c2 = cell + dir;
  if (c2 < 0 || c2 > i_last) return 0;
  const double a = uni_c(cmin, dc, c2), b = uni_c(cmin, dc, c2 + 1);
  const double fa = uni_f(m, a), fb = uni_f(m, b);
  if ((fa < 0.0) == (fb < 0.0)) return 0;
  *lo = a;
  *hi = b;
  *flo = fa;
  return 1;
}

/* refine.cuh:83-116 */
static double uni_bisect(const UniModel *m, double lo, double hi, double flo, int iters, double f_accept,
                         unsigned long long *stats) {
  for (int k = 0; k < iters; ++k) {
    const double mid = 0.5 * (lo + hi);
    const double fm = uni_f(m, mid);
    if ((fm < 0.0) == (flo < 0.0)) {
      lo = mid;
      flo = fm;
    } else {
      hi = mid;
    }
  }
  const double root = 0.5 * (lo + hi);
  if (f_accept < 1.0 && fabs(uni_f(m, root)) > f_accept) {
    ++stats[2];
    return NAN;
  }
  return root;
}

void mdo_uniform_refine(const float *row, int nc, const double *h, const double *vp, const double *vs,
                        const double *rho, int L, float period, int nmodes, double cmin, double cmax,
                        double c_tol_rel, double f_accept, double *out, unsigned *flags,
                        unsigned long long *stats) {
  const double dc = nc > 1 ? (cmax - cmin) / (double)(nc - 1) : 0.0;
  const double tol = c_tol_rel * cmin;
  int iters = 1; /* refine.cuh:38-45 */
  if (tol > 0.0 && dc > tol) {
    iters = (int)ceil(log2(dc / tol));
    if (iters < 1) iters = 1;
    if (iters > 60) iters = 60;
  }
  UniModel m = {h, vp, vs, rho, L, MDO_TWO_PI / (double)period};
  const double c_cap = vs[L - 1];
  int i_last = (int)((c_cap - cmin) / dc); /* scan_grid.hpp:19-24 */
  if (i_last > nc - 2) i_last = nc - 2;
  for (int target = 0; target < nmodes; ++target) {
    out[target] = NAN;
    int mode = 0, cell = -1, have_hidden = 0, n_point = 0;
    double h_lo = 0., h_hi = 0., h_flo = 0.;
    for (int i = 0; i + 1 < nc && i <= i_last && cell < 0 && !have_hidden;) {
      if ((row[i] < 0.0f) != (row[i + 1] < 0.0f)) {
        if (mode == target) {
          cell = i;
          break;
        }
        ++mode;
        ++i;
        continue;
      }
      const int tc = i + 1;
      int wlo = -1, whi = -1;
      if (tc >= 1 && tc + 1 < nc && tc <= i_last) {
        const float am = fabsf(row[tc - 1]), bm = fabsf(row[tc]), cm = fabsf(row[tc + 1]);
        const int no_sc_right = (row[tc] < 0.0f) == (row[tc + 1] < 0.0f);
        if (no_sc_right && am > bm && bm < cm && bm < 0.05f) {
          wlo = tc - 1;
          whi = tc + 1;
          ++n_point;
        }
      }
      if (wlo < 0) {
        ++i;
        continue;
      }
      const double c_a = uni_c(cmin, dc, wlo), c_b = uni_c(cmin, dc, whi), span = c_b - c_a;
      double prev_c = c_a, prev_f = uni_f(&m, c_a);
      for (int j = 1; j <= 65; ++j) {
        const double cj = c_a + span * (double)j / 65.0;
        const double fj = uni_f(&m, cj);
        if ((prev_f < 0.0) != (fj < 0.0)) {
          if (mode == target) {
            h_lo = prev_c;
            h_hi = cj;
            h_flo = prev_f;
            have_hidden = 1;
            break;
          }
          ++mode;
        }
        prev_c = cj;
        prev_f = fj;
      }
      i = whi;
    }
    stats[3] += (unsigned long long)n_point;
    double root = NAN;
    if (cell >= 0) {
      ++stats[0];
      const double lo = uni_c(cmin, dc, cell), hi = uni_c(cmin, dc, cell + 1);
      const double flo = uni_f(&m, lo), fhi = uni_f(&m, hi);
      if ((flo < 0.0) == (fhi < 0.0)) {
        ++stats[1];
        const int cl = cell - 1, cr = cell + 1;
        const int cand_l = cl >= 0 && ((row[cl] < 0.0f) == (row[cl + 1] < 0.0f));
        const int cand_r = cr + 1 < nc && cr <= i_last && ((row[cr] < 0.0f) == (row[cr + 1] < 0.0f));
        double llo = 0., lhi = 0., lflo = 0., rlo = 0., rhi = 0., rflo = 0.;
        const int left = cand_l && uni_retry(&m, cell, -1, i_last, cmin, dc, &llo, &lhi, &lflo);
        const int right = cand_r && uni_retry(&m, cell, +1, i_last, cmin, dc, &rlo, &rhi, &rflo);
        if (left != right) {
          ++stats[5];
          *flags |= 2u;
          root = left ? uni_bisect(&m, llo, lhi, lflo, iters, f_accept, stats)
                      : uni_bisect(&m, rlo, rhi, rflo, iters, f_accept, stats);
        } else {
          *flags |= 1u;
        }
      } else {
        root = uni_bisect(&m, lo, hi, flo, iters, f_accept, stats);
      }
    } else if (have_hidden) {
      ++stats[4];
      root = uni_bisect(&m, h_lo, h_hi, h_flo, iters, f_accept, stats);
    }
    if (root == root && root >= c_cap) root = NAN;
    out[target] = root;
  }
}
