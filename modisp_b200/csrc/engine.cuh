// engine.cuh -- device state and constants shared by the engine kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace md200 {

constexpr double TWO_PI = 6.283185307179586476925286766559;
constexpr unsigned FULL = 0xffffffffu;
constexpr int ROWS = 9;        // per-layer rows of the prepared table (7 used by the recurrence)
constexpr int EVAL_ROWS = 7;   // rows staged into shared memory for the recurrence
constexpr int SLOT = 5;        // doubles per bracket slot: lo, hi, flo, fhi, root
constexpr long long JMAX = 1LL << 22;  // scan points per trace before the workspace flag (default)
constexpr long long JMAX_FALLBACK = 1LL << 26;  // the fallback re-scan's limit

// Trace flag bits reported to the caller (values of python/modisp/__init__.py:15-32).
constexpr unsigned TRACE_SEARCH_UNCONVERGED = 4;
constexpr unsigned TRACE_WORKSPACE_LIMIT = 8;
constexpr unsigned TRACE_NEAR_CUTOFF = 16;
constexpr unsigned TRACE_NONFINITE = 32;
constexpr unsigned TRACE_REFINEMENT_FAILED = 64;
constexpr unsigned TRACE_F_REJECTED = 128;
constexpr unsigned TRACE_CLOSE_ROOT_RISK = 4096;
constexpr unsigned TRACE_ADAPTIVE_FALLBACK = 8192;
constexpr unsigned TRACE_FP64_REPAIR = 32768;
constexpr unsigned TRACE_CONTINUATION_APPROXIMATE = 65536;
// Engine-internal bits, cleared before the flags are written out.
constexpr unsigned INTERNAL_REPAIR = 1u << 28;
constexpr unsigned INTERNAL_MASK = 0xF0000000u;

// Group-velocity flags (python/modisp/__init__.py:46-52).
constexpr unsigned GROUP_MISSING_ROOT = 1;
constexpr unsigned GROUP_POLISH_FAILED = 2;
constexpr unsigned GROUP_ILL_CONDITIONED = 8;
constexpr unsigned GROUP_CLOSE_ROOT = 16;
constexpr unsigned GROUP_NONFINITE = 32;

// Search levels reported by this engine (the reference's ladder levels do not
// apply): 20 FP64 scan, 21 FP32 scan with FP64 refinement, 22 FP32 scan repaired
// by an FP64 re-scan, 23 continuation-predicted, 24 the FP64 fallback re-scan of
// a trace the first search could not finish; -3 no SH guide, -4 empty window.
constexpr int LEVEL_FP64 = 20, LEVEL_FP32 = 21, LEVEL_REPAIRED = 22, LEVEL_CONTINUATION = 23, LEVEL_FALLBACK = 24;

// Device counters (int) used by the work lists.
enum Counter {
  C_SCAN_CURSOR = 0, C_NTRACE, C_NREFINE, C_REFINE_BEGIN, C_NGROUP, C_REPAIR_CURSOR, C_NREPAIR,
  C_JFAIL, C_GROUP_BEGIN, C_NSUSPECT, C_REFINE_CURSOR, C_NTARGET, C_NCROOT,
  // split FP32 scan: active-list sizes by round parity, the trace-list feed
  // cursor, this round's fill base and count, FP64 re-evaluations, window
  // requests, the hand-over cursor
  C_SP_ACT0, C_SP_ACT1, C_SP_FEED, C_SP_BASE, C_SP_TAKE, C_SP_REDO, C_SP_ZOOM, C_SP_RESUME,
  C_COUNT
};

struct ScanState;
struct SplitSample;
struct SplitTrace;

struct Dev {
  // geometry of this run
  int B, Lmax, Ls, T, nmodes, K, KB, wave, fp32, nlog, nkmax, nsmax;
  int n_traces, group;
  long long jmax;   // scan points per trace before the workspace flag
  double tol, accept, close_rtol, density;
  // inputs (device)
  const double *h, *vp, *vs, *rho, *periods, *bounds_in;
  // prepared models
  int *mL, *mwater, *mstate;
  double *mlo, *mhi, *malpha;
  double *mtail;    // [B][2]: the two near-cutoff sample positions every scan that
                    // reaches the window end evaluates (hi, and vs_hs (1 - 1e-7))
  double4 *tail;    // [n_traces][2]: FP64 (c, F, g, log-magnitude) at those positions
  double *layer64;  // [B][ROWS][Ls]
  float *layer32;   // [B][ROWS][Ls]
  double4 *knot;    // [B][nkmax]: c, N(c), ln c, kink part of N over [c_i, c_i+1]
  int *nknot;
  double *seed;     // [B][nsmax]
  int *nseed;
  // trace geometry (filled by init_traces): model, period, output
  // index of mode 0, stride between modes, mode count.  Uniform batches: trace
  // t = b T + f, outputs [B][nmodes][T].  Ragged batches: traces in CSR order
  // (model b owns traces r_offsets[b] .. r_offsets[b+1]), outputs of model b a
  // [r_modes[b]][T_b] block at r_outbase[b].
  int ragged;
  const int *r_offsets, *r_modes;
  const long long *r_outbase;
  int *tr_model, *tr_stride, *tr_modes;
  double *tr_period;
  long long *tr_out;
  // traces
  int *nbr;
  unsigned *tflags;
  double *slot;     // [n_traces][KB][SLOT]
  int *trace_list, *repair_list, *refine_list, *group_list;
  int *ctr;
  // outputs
  double *vel;      // [B][nmodes][T]
  unsigned *oflags;
  int *olevels, *ocounts;
  double *grp;
  unsigned *gflags;
  double *gwin;     // [B][nmodes][T][2]
  double *bounds_out;  // [B][2] windows used (optional)
  unsigned *pred;      // [B][T] prediction flags (optional)
  unsigned char *cflags;  // [B][T] continuity-screen flags (optional; FP32-scan runs)
  double *cold;        // [n_traces][nmodes] roots of the screen's suspects before their FP64 re-scan
  int *ccount;         // [n_traces] root counts of those suspects before the re-scan
  // anchor continuation (engines created with it)
  signed char *crole;   // [n_traces]: 1 anchor, 2 target, 0 searched independently
  int *cleft, *cright;  // [n_traces]: a target's left and right anchor traces
  double *cslope;       // [n_traces][KB] dc/dln T at anchor roots
  unsigned char *csafe; // [n_traces] anchor roots usable as a source
  int *cont_list;       // target traces
  int *croot_list;      // predicted roots (trace * KB + rank)
  unsigned *ccode;      // [n_traces][KB] verdict of each predicted root
  // split FP32 scan (single-precision engines): rounds of positions, values,
  // FP64 re-evaluations, bookkeeping and trough windows over an active set of
  // traces; per-sample buffers [sp_cap][SPLIT_SAMPLES]
  int sp_cap;           // active-set capacity (traces)
  int *sp_act[2];       // active trace lists by round parity
  ScanState *sp_state;  // [n_traces] scan state between rounds
  struct SplitSample *sp_s;  // [sp_cap][SPLIT_SAMPLES] samples of the round
  struct SplitTrace *sp_tr;  // [sp_cap] the active traces' evaluation constants
  int *sp_kf;           // [n_traces] knot interval of the trace's next grid point (a lower bound)
  int *sp_redo;         // samples to evaluate in FP64
  int *sp_zoom;         // window requests: active-list index
  double *sp_zarg;      // [sp_cap][8] their arguments
  unsigned long long *stats;
};

// Continuity-screen flags (python/modisp/_continuity.py:6-14).
constexpr unsigned char CONT_REVIEWED = 1, CONT_REPAIRED = 2, CONT_UNRESOLVED = 4, CONT_NO_BILATERAL = 8,
                        CONT_ENVELOPE = 16, CONT_CLOSE_FP32 = 32, CONT_PREDICTION = 64;
// PredictionFlag.REVIEW (python/modisp/__init__.py:55-68).
constexpr unsigned PRED_REVIEW = 4096;

}  // namespace md200
