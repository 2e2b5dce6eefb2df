/*
 * md_oracle.h -- CPU restatement of modisp's FP64 dispersion numerics.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the test suite,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg compare the CUDA engine
 * against.  Nothing in the product (modisp_b200/) links, loads or calls it.
 *
 * Each function restates one reference routine; the citation names the
 * reference file and lines (paths relative to the modisp source tree).
 * Parity is pinned two ways (tests/test_oracle.py): bitwise against the
 * reference CPU engine compiled from its own sources into oracle/_ref/, and
 * against the golden vectors under tests/golden/.
 *
 * Units: km, km/s, g/cm^3, s, rad/s.  Models are [L] rows (h, vp, vs, rho);
 * the last row is the half-space (its thickness is ignored).
 */
#ifndef MD_ORACLE_H
#define MD_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

/* Normalized Dunkin P-SV secular value F and shape feature g
 * (cpp/common/dunkin.hpp:358-448, NORMALIZE=true, no omega clamp, as used by
 * md::evaluate / md::shape_evaluate in cpp/common/physics.hpp:60-82). */
double mdo_rayleigh(const double *h, const double *vp, const double *vs, const double *rho,
                    int L, double omega, double c, double *shape);

/* SH (Love) secular value and shape (cpp/common/physics.hpp:33-53). */
double mdo_love(const double *h, const double *vs, const double *rho,
                int L, double omega, double c, double *shape);

/* wave 0 = Rayleigh, 1 = Love; dispatch of cpp/common/physics.hpp:60-82. */
double mdo_secular(const double *h, const double *vp, const double *vs, const double *rho,
                   int L, int wave, double omega, double c, double *shape);

/* Unwrapped SH phase (cpp/common/love_phase.hpp:251-277); NaN where undefined. */
double mdo_love_phase(const double *h, const double *vs, const double *rho,
                      int L, double omega, double c);

/* Search window [lo, hi) of one model (cpp/cpu/solver.cpp:781-790 with
 * automatic_lower, cpp/common/physics.hpp:140-175). */
void mdo_bounds(const double *h, const double *vp, const double *vs, const double *rho,
                int L, int wave, double *lo, double *hi);

/* Brent-Dekker bracketed refinement (cpp/common/refinement.hpp:341-396). */
double mdo_refine(const double *h, const double *vp, const double *vs, const double *rho,
                  int L, int wave, double omega, double a, double b, double fa, double fb,
                  double tol, int *evaluations);

/* Dense-grid root search of one trace (cpp/cpu/solver.cpp:221-252 collect_roots and
 * :329-370 search_dense, factor 1, whole window at once).  Writes up to K ascending
 * roots; returns the count, or -1 when the grid is ambiguous. */
int mdo_dense_roots(const double *h, const double *vp, const double *vs, const double *rho,
                    int L, int wave, double period, double lo, double hi, int K, double tol,
                    double *roots);

/* Implicit derivatives of the secular function at (c, omega) by the complex-step
 * method in long double: writes dF/dk and dF/domega (k = omega/c).  Independent of
 * the CUDA engine's forward-mode derivatives. */
void mdo_derivatives(const double *h, const double *vp, const double *vs, const double *rho,
                     int L, int wave, double omega, double c, double *dfdk, double *dfdw);

/* Group velocity U = -F_k/F_omega after a long-double Brent polish of the root in
 * [lower, upper].  Returns 0 on success, nonzero if the polish fails. */
int mdo_group(const double *h, const double *vp, const double *vs, const double *rho,
              int L, int wave, double omega, double root, double lower, double upper,
              double *group);

/* dF/dtheta for every layer parameter (4*L values: h, vp, vs, rho blocks) and
 * dF/dc at fixed omega, by complex step in long double. */
void mdo_parameter_derivatives(const double *h, const double *vp, const double *vs,
                               const double *rho, int L, int wave, double omega, double c,
                               double *dfdtheta, double *dfdc);

/* Stage 2 of the legacy uniform-grid path for one (model, period) trace
 * (cpp/cuda/refine.cuh:131-317 and :33-116, cpp/cuda/refine.cu:233): each mode
 * m < nmodes walks the row of single-precision values `row` [nc] from the
 * start, as the reference's thread for mode m does, then confirms, relocates and
 * bisects its bracket in FP64.  `period` is the single-precision period the
 * reference stores.  Writes out[nmodes] (NaN where absent), ORs the trace flags
 * (1 unresolved, 2 relocated) into *flags and adds the six counters (brackets,
 * rejected_sign, rejected_f, troughs, hidden_roots, relocated) to stats. */
void mdo_uniform_refine(const float *row, int nc, const double *h, const double *vp, const double *vs,
                        const double *rho, int L, float period, int nmodes, double cmin, double cmax,
                        double c_tol_rel, double f_accept, double *out, unsigned *flags,
                        unsigned long long *stats);

#ifdef __cplusplus
}
#endif
#endif
