/*
 * modisp_b200.h -- C ABI of the B200 dispersion engine (libmodisp_b200.so).
 *
 * The engine is the drop-in for modisp's CUDA backend plugin: one engine object
 * per Solver, created with a capacity and a fixed geometry, run once per chunk,
 * closed when the Solver is.  Every entry point maps onto one item of the
 * reference plugin interface; the citation names the reference file:line it
 * replaces (paths relative to the modisp source tree).  All functions return 0
 * on success and a nonzero status on failure, with the message available from
 * md200_last_error() (the reference's legacy C ABI convention,
 * cpp/cuda/coarse_scan.cu:31-39).  No torch types cross this boundary.
 *
 * Arrays are C-contiguous: models [B, L] float64, periods [T], bounds [B, 2],
 * phase/group velocities [B, nmodes, T] (model, mode, period -- the reference
 * output layout, cpp/cuda/refine.cuh:168-172), trace arrays [B, T].
 */
#ifndef MODISP_B200_H
#define MODISP_B200_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

#define MD200_ABI_VERSION 3
/* Statistics written by md200_run (indices into the stats array). */
enum md200_stat {
  MD200_STAT_EVALUATIONS = 0,      /* secular evaluations, all precisions */
  MD200_STAT_EVALUATIONS_FP32 = 1, /* of which FP32 */
  MD200_STAT_LAYER_STEPS = 2,      /* layer recurrence steps, all evaluations */
  MD200_STAT_LAYER_STEPS_FP32 = 3,
  MD200_STAT_BRACKETS = 4,         /* sign-change brackets refined */
  MD200_STAT_PROBES = 5,           /* same-sign trough probes */
  MD200_STAT_PROBE_PAIRS = 6,      /* probes that split a hidden root pair */
  MD200_STAT_REPAIR_TRACES = 7,    /* FP32 traces re-scanned in FP64 */
  MD200_STAT_UNCONVERGED = 8,      /* traces reported unconverged */
  MD200_STAT_GROUP_ROOTS = 9,      /* group velocities computed */
  MD200_STAT_ROOTS = 10,           /* finite phase velocities returned */
  MD200_STAT_TRACES = 11,          /* traces searched */
  MD200_STAT_DUAL_LAYER_STEPS = 12,/* layer steps of forward-mode derivative evaluations */
  MD200_STAT_CONT_ACCEPTED = 13,   /* continuation targets accepted */
  MD200_STAT_CONT_FALLBACK = 14,   /* continuation targets searched globally */
  MD200_STAT_CONTINUITY = 15,      /* FP32-scan traces re-scanned by the continuity recheck */
  MD200_STAT_FALLBACK = 16,        /* traces re-scanned by the FP64 fallback (first search unfinished) */
  MD200_STAT_CONT_ANCHORS = 17,    /* continuation anchor traces */
  MD200_STAT_CONT_EVALUATIONS = 18,/* secular evaluations of continuation targets (prediction + audit) */
  MD200_STAT_SPLIT_EVAL_STEPS = 19,/* FP32 layer steps of the split scan's evaluation kernel (every
                                      sample it evaluated, those past a trace's last bracket too) */
  MD200_STAT_COUNT = 20
};

typedef struct md200_engine md200_engine;

/* Engine configuration; the fields mirror the positional arguments of the
 * reference QeSolver constructor (cpp/cuda/qe.cu:978, called from
 * python/modisp/__init__.py:398-400) plus the engine's own tuning knobs. */
typedef struct md200_options {
  int accuracy;            /* 0 high, 1 balanced, 2 fast, 4 auto (recorded; the scan rule is the same) */
  double period_threshold; /* accepted for compatibility */
  double close_root_rtol;  /* close-root threshold, default 0.005 */
  int shape;               /* accepted for compatibility */
  double sampling_rtol;    /* accepted for compatibility */
  int secular;             /* 0 dunkin, 1 fast: one compound-matrix evaluator serves both */
  int refinement;          /* 1 Brent (the engine's refinement); 0 and 2 are accepted */
  int love_phase;          /* accepted for compatibility */
  int single_precision;    /* 1: FP32 scan + FP64 refinement; 0: FP64 throughout */
  int group_velocity;      /* 1: FP64 group velocity from implicit derivatives */
  double group_rtol;       /* accepted for compatibility (the derivative is analytic) */
  int continuation;        /* 1: anchor continuation over sorted unique periods */
  int anchor_stride;       /* anchor spacing in periods (>= 2) */
  double scan_density;     /* scan points per phase unit; <= 0 selects the default */
  int log_points;          /* background log-spaced points per window; <= 0 default */
  int warps_per_block;     /* scan CTA shape; <= 0 default */
  int blocks_per_sm;       /* persistent CTAs per SM; <= 0 default */
  int continuity_check;    /* FP32 scan: the reference's continuity screen on the results
                              (cpp/cpu/continuity_screen.hpp:8-67) and an FP64 re-scan of
                              its suspects (default 1) */
  long long scan_points;   /* scan points per trace before TRACE_WORKSPACE_LIMIT in the first
                              search (<= 0: 2^22); an unfinished trace is re-scanned in FP64
                              with a limit of 2^26 (TRACE_ADAPTIVE_FALLBACK, level 24) */
  int scan_mode;           /* FP32 scan: 0 auto (rounds of split kernels for Rayleigh runs of
                              4096 traces or more, else the fused one-warp-per-trace
                              kernel), 1 fused, 2 split; all return the same brackets bit
                              for bit */
} md200_options;

/* Fill *options with the defaults of a high-accuracy FP64 engine. */
void md200_default_options(md200_options *options);

/* Replaces QeSolver(B, L, nf, nmodes, ...) (cpp/cuda/qe.cu:978-1036).  capacity is
 * the maximum number of models per run; layers, periods, nmodes fix the
 * geometry.  Returns NULL on failure. */
md200_engine *md200_create(int device, int capacity, int layers, int periods, int nmodes,
                           const md200_options *options);

/* Replaces QeSolver.run(...) (cpp/cuda/qe.cu:1060-1119) with host arrays: copies
 * inputs to the device, solves, copies outputs back and synchronises.
 *   thickness, vp, vs, rho : [models, layers]
 *   periods                : [periods]
 *   bounds                 : [models, 2] search windows [lo, hi), or NULL to compute
 *                            them on the device (cpp/cpu/solver.cpp:781-790).  A
 *                            non-positive lo asks for the automatic lower bound;
 *                            hi is capped below the half-space shear velocity.
 *   wave                   : 0 Rayleigh, 1 Love
 * Outputs (NULL to skip the optional ones):
 *   velocity [models, nmodes, periods] float64 (NaN where no root)
 *   flags, levels, counts [models, periods]
 *   group, group_flags [models, nmodes, periods] (engine created with group_velocity)
 *   prediction_flags [models, periods] (engine created with continuation)
 *   continuity_flags [models, periods] uint8: the continuity screen's flags
 *                            (python/modisp/_continuity.py:6-14; the reference
 *                            returns them as DispersionBatch.continuity_flags,
 *                            python/modisp/__init__.py:424-431): REVIEWED 1,
 *                            REPAIRED 2, UNRESOLVED 4, NO_BILATERAL 8, ENVELOPE 16,
 *                            CLOSE_FP32 32, PREDICTION 64.  The screen runs in
 *                            FP32-scan engines with continuity_check; other
 *                            engines write 0 (unscreened).
 *   bounds_out [models, 2] the windows searched
 *   stats [nstats] counters, see enum md200_stat. */
int md200_run(md200_engine *engine, const double *thickness, const double *vp, const double *vs,
              const double *rho, int models, const double *periods, const double *bounds,
              double c_tol_rel, double f_accept, int wave, double *velocity, unsigned *flags,
              int *levels, int *counts, double *group, unsigned *group_flags,
              unsigned *prediction_flags, uint8_t *continuity_flags, double *bounds_out,
              unsigned long long *stats, int nstats);

/* As md200_run, but every array is a device pointer and the work is enqueued on
 * `stream` (a cudaStream_t; NULL selects the engine's own stream, cudaStreamLegacy the
 * legacy default stream) without a host
 * synchronisation.  stats, if given, is a device array of MD200_STAT_COUNT
 * counters. */
int md200_run_device(md200_engine *engine, const double *thickness, const double *vp,
                     const double *vs, const double *rho, int models, const double *periods,
                     const double *bounds, double c_tol_rel, double f_accept, int wave,
                     double *velocity, unsigned *flags, int *levels, int *counts, double *group,
                     unsigned *group_flags, unsigned *prediction_flags, uint8_t *continuity_flags,
                     double *bounds_out, unsigned long long *stats, void *stream);

/* Ragged batch (no counterpart in the reference, whose periods are one array
 * shared by every model, python/modisp/__init__.py:285-286; its per-row form
 * allows one period per model only, cpp/cuda/qe.cu:1069-1070): every model has
 * its own period list and its own mode count, and all of them share one set of
 * launches.  Host arrays, waits for the result.
 *   period_offsets [models + 1] : model b's periods are periods[period_offsets[b] ..
 *                                 period_offsets[b+1]) (CSR; offsets[0] = 0,
 *                                 non-decreasing; the total is at most capacity x
 *                                 the engine's periods)
 *   modes [models]              : mode count of model b, 1 .. the engine's nmodes
 *   bounds [models, 2]          : search windows as in md200_run, or NULL (automatic)
 * Outputs: per trace (CSR order) flags, levels, counts, continuity_flags
 * [traces]; velocity (and group, group_flags) hold, for model b, a [modes[b]][T_b]
 * block (mode, period),
 * the blocks concatenated in model order (sum of modes[b] T_b values).
 * Trace semantics are those of md200_run. */
int md200_run_ragged(md200_engine *engine, const double *thickness, const double *vp, const double *vs,
                     const double *rho, int models, const int *period_offsets, const double *periods,
                     const int *modes, const double *bounds, double c_tol_rel, double f_accept, int wave,
                     double *velocity,
                     unsigned *flags, int *levels, int *counts, double *group, unsigned *group_flags,
                     uint8_t *continuity_flags, unsigned long long *stats, int nstats);

/* Device-pointer form of md200_run_ragged, enqueued on `stream` (NULL = the
 * engine's stream) without a host synchronisation.  `traces` is
 * period_offsets[models]; out_offsets [models] gives the index of model b's
 * output block (the running sum of modes[b'] T_b' over b' < b).  The CSR
 * description is not checked on the device: offsets must be non-decreasing and
 * the output arrays large enough; mode counts are clamped to 1 .. nmodes. */
int md200_run_ragged_device(md200_engine *engine, const double *thickness, const double *vp,
                            const double *vs, const double *rho, int models, int traces,
                            const int *period_offsets, const double *periods, const int *modes,
                            const long long *out_offsets, const double *bounds, double c_tol_rel,
                            double f_accept, int wave,
                            double *velocity, unsigned *flags, int *levels, int *counts, double *group,
                            unsigned *group_flags, uint8_t *continuity_flags, unsigned long long *stats,
                            void *stream);

/* CUDA-graph capture of device-pointer runs (no counterpart in the reference,
 * which launches its stages one by one, cpp/cuda/qe.cu:927-957).  Between
 * md200_graph_begin and md200_graph_end, md200_run_device and
 * md200_run_ragged_device calls made with stream NULL are recorded on the
 * engine's stream instead of executed (one or more calls, e.g. both waves); the
 * recorded launches read the device pointers given at capture, so a replay
 * solves whatever those buffers hold at launch time.  md200_graph_launch
 * replays the graph on `stream` (NULL = the engine's stream).  Stage times are
 * not recorded inside a graph.  A new capture replaces the previous graph. */
int md200_graph_begin(md200_engine *engine);
int md200_graph_end(md200_engine *engine);
int md200_graph_launch(md200_engine *engine, void *stream);

/* Phase- and group-velocity Jacobians of solved roots (no counterpart in the
 * reference, which returns no derivatives; they serve the gradient of a misfit
 * between predicted and observed dispersion).  For every finite root
 * velocity[b][mode][period] of models [models][layers] (the engine's geometry)
 * at `periods`, jac_phase[b][mode][period][4][layers] receives dc/dm and
 * jac_group (optional) dU/dm, with m the row's thickness, vp, vs, rho in that
 * order (km/s per km, per km/s, per g/cc).  The layer tables are prepared again
 * from the inputs; dc/dm = (c/k) F_m / F_k and dU/dm from the second
 * derivatives of the secular function, by a forward (k, omega) sweep and an
 * adjoint sweep through the layer recurrence (adjoint.cuh).  Rows of zero
 * thickness (padding) and the half-space thickness get 0; NaN rows mark a
 * missing root (or, for jac_group, a missing group velocity where `group` is
 * given) or a root with F_k = 0 or F_omega = 0.  Models of up to 265 rows.
 * Device pointers, enqueued on `stream` (NULL = the engine's stream). */
int md200_jacobian_device(md200_engine *engine, const double *thickness, const double *vp,
                          const double *vs, const double *rho, int models, const double *periods,
                          int wave, const double *velocity, const double *group, double *jac_phase,
                          double *jac_group, void *stream);

/* Host-pointer form of md200_jacobian_device (waits for the result);
 * `failed` (optional) receives the number of finite roots whose rows are NaN. */
int md200_jacobian(md200_engine *engine, const double *thickness, const double *vp, const double *vs,
                   const double *rho, int models, const double *periods, int wave,
                   const double *velocity, const double *group, double *jac_phase,
                   double *jac_group, int *failed);

/* Vector-Jacobian product without forming the Jacobians (no counterpart in the
 * reference): grad[4][models][layers] = sum over cells of
 * weight_phase[cell] dc/dm + weight_group[cell] dU/dm (either weight array may
 * be NULL; cells without a finite root, or without a finite `group` where it is
 * given, contribute nothing).  The backward pass of a misfit: weights are the
 * misfit's derivatives with respect to each phase and group velocity.
 * Accumulated with atomic adds: the summation order, and so the last bits, may
 * differ between calls.  Device pointers, enqueued on `stream`. */
int md200_vjp_device(md200_engine *engine, const double *thickness, const double *vp,
                     const double *vs, const double *rho, int models, const double *periods,
                     int wave, const double *velocity, const double *group,
                     const double *weight_phase, const double *weight_group, double *grad,
                     void *stream);

/* Host-pointer form of md200_vjp_device (waits for the result). */
int md200_vjp(md200_engine *engine, const double *thickness, const double *vp, const double *vs,
              const double *rho, int models, const double *periods, int wave,
              const double *velocity, const double *group, const double *weight_phase,
              const double *weight_group, double *grad);

/* Device time (ms) of each stage of the engine's last run, from cudaEvent pairs
 * recorded on the run's stream (the reference's profile timings,
 * cpp/cuda/qe.cu:853-864): [0] model preparation, [1] trace list, [2] scan,
 * [3] refinement, [4] repair selection, [5] FP64 re-scan, [6] re-scan
 * refinement, [7] assembly, [8] group velocity, [9] FP64 continuity recheck
 * (screen, re-scan, refinement, assembly and group velocity of the suspects),
 * [10] the split scan's evaluation kernel alone (its launches summed; 0 when the
 * run used the fused scan).  Waits for the run to finish. */
int md200_stage_times(md200_engine *engine, double *ms, int n);

/* Number of kernel launches the engine's last run enqueued (counted as it
 * launched them); before any run, those of a run without continuity flags. */
int md200_kernel_launches(md200_engine *engine);

/* Replaces QeSolver.close() (cpp/cuda/qe.cu:1039-1059). */
void md200_destroy(md200_engine *engine);

/* Message of the last failure on this thread (static storage). */
const char *md200_last_error(void);

/* Module functions of the plugin (cpp/cuda/qe.cu:1131-1142): */
int md200_device_count(void);                 /* number of CUDA devices, 0 if none */
int md200_available(int device);              /* 1 when `device` is a usable sm_100 GPU */
int md200_set_device(int device);
int md200_memory_info(size_t *free_bytes, size_t *total_bytes);
int md200_device_name(int device, char *name, int length);

/* Kernel attributes of the engine's kernels (cpp/cuda/qe.cu:1143-1164): writes a
 * JSON object describing registers, shared memory and occupancy to `json`. */
int md200_kernel_report(int layers, int single_precision, char *json, int length);

/* Measurement helper with no counterpart in the reference: sustained non-tensor
 * FMA throughput of `device` in flop/s (FMA = 2), FP64 when fp64 != 0 else FP32
 * -- the roofline denominator for the engine's CUDA-core kernels. */
int md200_measure_peak(int device, int fp64, double *flops);

/* The continuity screen alone, on host arrays: replaces the reference's
 * continuity_screen module function (cpp/cpu/continuity_screen.hpp:8-67, bound at
 * cpp/cpu/solver.cpp:775-777).  periods [T], velocity [B, K, T] float64 (pass
 * float32 results widened, with single = 1, for the reference's float32 screen:
 * values compared as float32 and the 16-ULP CLOSE_FP32 rule on), prediction
 * [B, T] or NULL, bilateral = the envelope rule on.  Outputs flags [B, T] (the
 * ENVELOPE 16, CLOSE_FP32 32, PREDICTION 64 and NO_BILATERAL 8 bits) and
 * *suspect = 1 when any trace has one of the first three. */
int md200_continuity_screen(int device, const double *periods, int T, const double *velocity, int B, int K,
                            const uint32_t *prediction, int single, int bilateral, uint8_t *flags,
                            int *suspect);

/* Group velocities of one model's known ordered roots (guards included), for a
 * trace repaired outside the engine: replaces the plugin's _review_groups
 * (cpp/common/review_groups.hpp:9-63, cpp/cuda/review_groups.cu:6-35).  Host
 * arrays: one model [layers], roots [known]; outputs [modes].  A root without a
 * slot is MISSING_ROOT (1), a close pair CLOSE_ROOT (16). */
int md200_group_roots(const double *thickness, const double *vp, const double *vs,
                      const double *rho, int layers, int wave, double period,
                      const double *roots, int known, int modes, double close_rtol,
                      double *group, unsigned *group_flags);

/* ---- Cross-period mode-reliability checks ------------------------------ *
 * Replace check_mode_reliability (python/modisp/reliability.py:49-145): flags
 * [B][K][T] (ModeReliabilityFlag bits, :12-24) and an "assessed" mask for a
 * result's phase velocities, without editing them.  The period order is a plan
 * of T entries (stable sort, distinct periods, gaps, prediction ratios); the
 * Python layer builds it with the reference's own numpy arithmetic, and
 * md200_reliability_plan builds it in C (libm log / log1p, which can differ from
 * numpy's in the last bit of a ratio). */
#define MD200_PLAN_FIRST 1     /* first period in sorted order: unassessed */
#define MD200_PLAN_DUPLICATE 2 /* equal to the previous distinct period */
#define MD200_PLAN_GAP 4       /* log gap to the previous period above the limit */
#define MD200_PLAN_PREDICT 8   /* linear prediction from the two previous periods */
typedef struct {
  int32_t prev;      /* previous distinct period (index into periods), -1 for the first */
  int32_t older;     /* the distinct period before prev, when MD200_PLAN_PREDICT */
  int32_t kind;      /* MD200_PLAN_* bits */
  int32_t dup_begin; /* a distinct period's duplicates are order[dup_begin .. dup_end) */
  int32_t dup_end;
  int32_t reserved;
  double ratio;      /* log_gap(prev, t) / log_gap(older, prev), when MD200_PLAN_PREDICT */
} md200_period_plan;

/* Plan for periods[T] (finite, positive): plan[T], order[T] (stable sort).
 * reliability.py:7-9 (log gap) and :107-144 (period walk). */
int md200_reliability_plan(const double *periods, int T, double max_log_period_gap,
                           md200_period_plan *plan, int32_t *order);

/* The checks on host arrays: velocity [B][K][T] (positive or NaN), trace_flags
 * [B][T] (NULL: none), root_count [B][T] (NULL: finite roots per trace), plan and
 * order from a plan builder.  Outputs flags [B][K][T] (uint16) and assessed
 * [B][K][T] (0/1).  Device buffers are allocated and freed on a private stream. */
int md200_mode_reliability(int device, const double *velocity, const uint32_t *trace_flags,
                           const int64_t *root_count, int B, int K, int T,
                           const md200_period_plan *plan, const int32_t *order,
                           double close_root_rtol, double max_relative_step, double prediction_rtol,
                           uint16_t *flags, uint8_t *assessed);

/* The same on device buffers (velocity, trace_flags, root_count, flags, assessed;
 * plan and order stay host arrays), enqueued on `stream` (NULL: the legacy
 * stream) and not waited for.  The plan is uploaded to stream-ordered scratch. */
int md200_mode_reliability_device(const double *velocity, const uint32_t *trace_flags,
                                  const int64_t *root_count, int B, int K, int T,
                                  const md200_period_plan *plan, const int32_t *order,
                                  double close_root_rtol, double max_relative_step,
                                  double prediction_rtol, uint16_t *flags, uint8_t *assessed,
                                  void *stream);

/* The same with the plan and order already on the device (from a plan
 * uploaded once for many checks with the same periods): only the kernel is
 * enqueued.  The plan's indices are trusted: build it with a plan builder. */
int md200_mode_reliability_planned(const double *velocity, const uint32_t *trace_flags,
                                   const int64_t *root_count, int B, int K, int T,
                                   const md200_period_plan *plan, const int32_t *order,
                                   double close_root_rtol, double max_relative_step,
                                   double prediction_rtol, uint16_t *flags, uint8_t *assessed,
                                   void *stream);

/* md200_group_roots without any device allocation.  No counterpart in the
 * reference: it exists for callers that cannot call cudaMalloc -- code whose GPU
 * memory is owned by another allocator (a framework's caching allocator that has
 * reserved the device), and repair loops that must not pay the device-wide
 * synchronisation of cudaFree on every trace.  Same arguments and results as
 * md200_group_roots; the scratch is a static 16 KiB device array (2048 doubles,
 * held by every GPU that loads the library until exit) that must hold
 * 7*layers + known + modes + ceil(modes/2) doubles (e.g. 256 layers with up to
 * 100 roots and modes); larger requests fail with a message and touch nothing.
 * Every call looks up the array's address on the current device
 * (cudaGetSymbolAddress), so a device reset between calls does no harm.  Its
 * copies are synchronous (cudaMemcpy) and its kernel runs on the legacy default
 * stream.  Calls share the array, which keeps the last call's contents (each
 * call rewrites what it reads): calls that overlap on the GPU (from several host
 * threads, or processes sharing a context) race. */
int md200_group_roots_static(const double *thickness, const double *vp, const double *vs,
                             const double *rho, int layers, int wave, double period,
                             const double *roots, int known, int modes, double close_rtol,
                             double *group, unsigned *group_flags);

/* ---------------------------------------------------------------------------
 * Legacy uniform-grid Rayleigh path (the reference's search_strategy="uniform",
 * python/modisp/_legacy.py:124-431, bound as the plugin classes CoarseScan and
 * Refine of cpp/cuda/bindings.cpp:121-345).  One object type serves both of the
 * reference's stage states: a scan object (md200_uniform_grid with nmodes = 0)
 * holds FP32 secular values on the grid c_i = cmin + i (cmax - cmin) / (nc - 1)
 * per (model, period); a refinement object (nmodes > 0) reads a scan object's
 * values and holds roots [models][nmodes][periods] (NaN where a mode is
 * missing), per-trace flags (1 unresolved bracket, 2 relocated bracket) and six
 * counters (brackets, rejected_sign, rejected_f, troughs, hidden_roots,
 * relocated).  Solid models only (every vs > 0); periods are kept in single
 * precision as the reference keeps them.  Work is enqueued on the legacy default
 * stream (so calls on different objects are ordered); copies to the host wait
 * for it.  Errors return 1 with md200_last_error(); numerical problems are
 * flags and NaN, never errors.
 * ------------------------------------------------------------------------- */
typedef struct md200_uniform md200_uniform;

/* Replaces md_cuda_create (cpp/cuda/coarse_scan.cu:63) and md_refine_create
 * (cpp/cuda/refine.cu:48): B models of L rows (layers plus half-space, L >= 2). */
md200_uniform *md200_uniform_create(int models, int layers);

/* Replaces md_cuda_upload_models (coarse_scan.cu:89) / md_refine_upload_models
 * (refine.cu:73): four [B][L] arrays; zero-thickness rows are identity steps. */
int md200_uniform_models(md200_uniform *u, const double *thickness, const double *vp, const double *vs,
                         const double *rho);

/* Replaces md_cuda_upload_periods (coarse_scan.cu:111) / md_refine_upload_periods
 * (refine.cu:94); a different period count drops the allocated outputs. */
int md200_uniform_periods(md200_uniform *u, int periods, const double *values);

/* Replaces md_cuda_set_output (coarse_scan.cu:150; nmodes = 0, nc >= 1) and
 * md_refine_set_output (refine.cu:138; nmodes >= 1, nc >= 2). */
int md200_uniform_grid(md200_uniform *u, int nc, int nmodes);

/* Replaces md_cuda_run (coarse_scan.cu:183): enqueue the FP32 values over
 * [cmin, cmax]; cells past the half-space shear velocity's last cell are NaN. */
int md200_uniform_scan(md200_uniform *u, double cmin, double cmax);

/* Replaces md_cuda_download (coarse_scan.cu:252): float [B][periods][nc]. */
int md200_uniform_rows(md200_uniform *u, float *rows);

/* Stage 1 values from the caller instead of md200_uniform_scan: float
 * [B][periods][nc] as md200_uniform_rows returns them, taken as a scan over
 * [cmin, cmax].  No counterpart in the reference (whose refinement reads only its
 * own scan's device buffer, cpp/cuda/bindings.cpp:263-279); it lets stage 2 run
 * on values computed elsewhere, such as another implementation's stage 1. */
int md200_uniform_set_rows(md200_uniform *u, const float *rows, double cmin, double cmax);

/* Replaces md_refine_run (refine.cu:191): enqueue stage 2 on `scan`'s values
 * (same B, L, periods and nc; the range its last md200_uniform_scan ran with).
 * nmodes 0 keeps the allocated count; c_tol_rel sets the bisection count
 * (md200_uniform_iterations), f_accept < 1 rejects roots with |F| above it. */
int md200_uniform_refine(md200_uniform *u, const md200_uniform *scan, double cmin, double cmax,
                         double c_tol_rel, double f_accept, int nmodes);

/* Replaces md_cuda_sync / md_refine_sync (coarse_scan.cu:225, refine.cu:256). */
int md200_uniform_sync(void);

/* Replace md_refine_download (refine.cu:262), md_refine_flags (refine.cu:376)
 * and md_refine_stats (refine.cu:291; n >= 6). */
int md200_uniform_velocity(md200_uniform *u, double *velocity);
int md200_uniform_flags(md200_uniform *u, uint32_t *flags);
int md200_uniform_stats(md200_uniform *u, uint64_t *stats, int n);

/* Replaces md_refine_iters_for (refine.cu:333): bisections for a cell of width
 * dc to reach c_tol_rel * cmin (1..60). */
int md200_uniform_iterations(double dc, double c_tol_rel, double cmin);

/* Replaces md_cuda_kernel_report / md_refine_kernel_report (coarse_scan.cu:279,
 * refine.cu:337): stage 0 the scan kernel, 1 the bisection kernel. */
int md200_uniform_kernel_report(int stage, int layers, int block, char *text, int length);

/* Replaces md_cuda_free / md_refine_free. */
void md200_uniform_destroy(md200_uniform *u);

#ifdef __cplusplus
}
#endif
#endif
