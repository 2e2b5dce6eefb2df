// engine.cu -- host orchestration and C ABI of the modisp_b200 engine.
//
// One engine per Solver (the reference's QeSolver contract, cpp/cuda/qe.cu:836-1170):
// device workspace sized at creation for a capacity of models, one stream, all
// stages enqueued back to back with device-side work lists so a run needs no
// host synchronisation until its outputs are read.
#include <cuda_runtime.h>

#include <algorithm>
#include <exception>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "modisp_b200.h"
#include "kernels.cuh"
#include "adjoint.cuh"
#include "reliability.cuh"
#include "continuation.cuh"
#include "split_scan.cuh"
#include "uniform.cuh"

using namespace md200;

namespace {

thread_local std::string g_error;

int fail(const std::string &msg) {
  g_error = msg;
  return 1;
}

// An exception caught at a C entry point (host allocation failure or a thread
// that could not start) becomes an error status: none may cross the C ABI.
int fail_exception() {
  try {
    throw;
  } catch (const std::bad_alloc &) {
    g_error = "modisp_b200: out of host memory";
  } catch (const std::exception &ex) {
    g_error = std::string("modisp_b200: ") + ex.what();
  } catch (...) {
    g_error = "modisp_b200: internal error";
  }
  return 1;
}

#define MD200_CK(call)                                                                     \
  do {                                                                                     \
    cudaError_t err__ = (call);                                                            \
    if (err__ != cudaSuccess)                                                              \
      return fail(std::string("modisp_b200 CUDA: ") + cudaGetErrorString(err__) + " (" +  \
                  #call + ")");                                                            \
  } while (0)

// Host copies between pinned staging and the caller's arrays, spread over up to
// `max_threads` threads (8 while the GPU still works, more when nothing else is
// left): the caller's output arrays are usually fresh (first-touch page faults)
// and a single core copies them at a fraction of the memory bandwidth.
struct HostCopy {
  void *dst;
  const void *src;
  size_t bytes;
};
void parallel_copy(const std::vector<HostCopy> &jobs, unsigned max_threads = 8) {
  size_t total = 0;
  for (const HostCopy &j : jobs) total += j.bytes;
  const unsigned hw = std::thread::hardware_concurrency();
  const unsigned nth = static_cast<unsigned>(std::min<size_t>(std::min(max_threads, hw ? hw : 1u), total >> 21));
  auto part = [&](size_t lo, size_t hi) {  // byte range [lo, hi) of the jobs laid end to end
    size_t off = 0;
    for (const HostCopy &j : jobs) {
      const size_t a = std::max(lo, off), b = std::min(hi, off + j.bytes);
      if (a < b) std::memcpy(static_cast<char *>(j.dst) + (a - off), static_cast<const char *>(j.src) + (a - off), b - a);
      off += j.bytes;
    }
  };
  if (nth <= 1) {
    part(0, total);
    return;
  }
  std::vector<std::thread> pool;
  unsigned started = 1;
  try {  // no exception may leave a C entry point: ranges without a thread are copied here
    pool.reserve(nth - 1);
    for (; started < nth; ++started) pool.emplace_back(part, total * started / nth, total * (started + 1) / nth);
  } catch (...) {
  }
  part(0, total / nth);
  for (unsigned t = started; t < nth; ++t) part(total * t / nth, total * (t + 1) / nth);
  for (std::thread &th : pool) th.join();
}

template <class T>
cudaError_t dalloc(T **p, size_t count) {
  *p = nullptr;
  if (count == 0) count = 1;
  return cudaMalloc(reinterpret_cast<void **>(p), count * sizeof(T));
}

}  // namespace

struct md200_engine {
  int device = 0, cap = 0, L = 0, T = 0, nmodes = 0;
  md200_options o{};
  cudaStream_t stream = nullptr;
  Dev d{};
  int sortcap = 0, prep_warps = 4, scan_warps = 4, scan_blocks64 = 0, scan_blocks32 = 0;
  int list_blocks = 0;
  size_t scan_smem64 = 0, scan_smem32 = 0, prep_smem = 0;
  // host-path buffers
  double *in_h = nullptr, *in_vp = nullptr, *in_vs = nullptr, *in_rho = nullptr,
         *in_per = nullptr, *in_bounds = nullptr;
  double *out_vel = nullptr, *out_grp = nullptr;
  unsigned *out_flags = nullptr, *out_gflags = nullptr, *out_pred = nullptr;
  unsigned char *out_cflags = nullptr;
  int *out_levels = nullptr, *out_counts = nullptr;
  unsigned long long *d_stats = nullptr;
  unsigned char *pinned = nullptr;
  size_t pinned_bytes = 0;
  // host-path Jacobian buffers (allocated on first use)
  double *jac_c = nullptr, *jac_u = nullptr, *jac_w = nullptr, *jac_grad = nullptr;
  // host-path ragged buffers (allocated on first use)
  int *rg_offsets = nullptr, *rg_modes = nullptr;
  long long *rg_outbase = nullptr;
  double *rg_periods = nullptr;
  std::vector<void *> owned;
  // host-path pipelining: chunks of models solved on `stream`, each chunk's outputs
  // copied back on `copy_stream` once its solve has ended (solved_ev) while the next
  // chunk is solved; chunk_ev marks the end of a chunk's copies
  static constexpr int MAX_CHUNKS = 8;
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t solved_ev[MAX_CHUNKS] = {};
  cudaEvent_t chunk_ev[MAX_CHUNKS] = {};
  // per-stage timing (cudaEvent pairs on the run's stream)
  static constexpr int NSTAGE = 10;
  cudaEvent_t ev[NSTAGE + 1] = {};
  // the split scan's evaluation launches, one event pair per round
  static constexpr int MAX_SPLIT_ROUNDS = 64;
  cudaEvent_t sp_ev[2 * MAX_SPLIT_ROUNDS] = {};
  int sp_timed = 0;  // rounds timed by the last run
  bool profiling = false;
  int last_launches = -1;  // kernels launched by the last run (enqueue)
  // CUDA graph of the calls captured between md200_graph_begin and md200_graph_end
  bool capturing = false;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
};

namespace {

template <class T>
int own_alloc(md200_engine *e, T **p, size_t count) {
  MD200_CK(dalloc(p, count));
  e->owned.push_back(*p);
  return 0;
}

void release(md200_engine *e) {
  if (!e) return;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(e->device);
  if (e->stream) cudaStreamSynchronize(e->stream);
  if (e->copy_stream) cudaStreamSynchronize(e->copy_stream);
  for (void *p : e->owned) cudaFree(p);
  e->owned.clear();
  if (e->pinned) cudaFreeHost(e->pinned);
  for (auto &x : e->ev)
    if (x) cudaEventDestroy(x);
  for (auto &x : e->chunk_ev)
    if (x) cudaEventDestroy(x);
  for (auto &x : e->solved_ev)
    if (x) cudaEventDestroy(x);
  for (auto &x : e->sp_ev)
    if (x) cudaEventDestroy(x);
  if (e->graph_exec) cudaGraphExecDestroy(e->graph_exec);
  if (e->graph) cudaGraphDestroy(e->graph);
  if (e->stream) cudaStreamDestroy(e->stream);
  if (e->copy_stream) cudaStreamDestroy(e->copy_stream);
  cudaSetDevice(prev);
}

size_t scan_smem(int warps, int Ls, size_t elem) {
  const size_t tab = (static_cast<size_t>(EVAL_ROWS) * Ls * elem + 15) & ~size_t(15);
  return static_cast<size_t>(warps) * (tab + 32 * sizeof(double));
}

int setup(md200_engine *e) {
  MD200_CK(cudaSetDevice(e->device));
  MD200_CK(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
  MD200_CK(cudaStreamCreateWithFlags(&e->copy_stream, cudaStreamNonBlocking));
  const int B = e->cap, L = e->L, T = e->T, nm = e->nmodes;
  Dev &d = e->d;
  d.Lmax = L;
  d.Ls = (L + 3) & ~3;
  d.T = T;
  d.nmodes = nm;
  d.K = nm + 2;
  d.KB = d.K;
  d.nlog = e->o.log_points > 0 ? e->o.log_points : 128;
  d.density = e->o.scan_density > 0. ? e->o.scan_density : 16.;
  d.nkmax = d.nlog + 1 + 2 * L;
  d.nsmax = 6 * L + 32;
  d.close_rtol = e->o.close_root_rtol > 0. ? e->o.close_root_rtol : .005;
  d.jmax = e->o.scan_points > 0 ? std::min<long long>(e->o.scan_points, JMAX_FALLBACK) : JMAX;
  d.fp32 = e->o.single_precision ? 1 : 0;
  d.group = e->o.group_velocity ? 1 : 0;
  const size_t nt = static_cast<size_t>(B) * T;
  if (own_alloc(e, &d.mL, B) || own_alloc(e, &d.mwater, B) || own_alloc(e, &d.mstate, B) ||
      own_alloc(e, &d.mlo, B) || own_alloc(e, &d.mhi, B) || own_alloc(e, &d.malpha, B) ||
      own_alloc(e, &d.mtail, 2 * static_cast<size_t>(B)) || own_alloc(e, &d.tail, 2 * nt) ||
      own_alloc(e, &d.layer64, static_cast<size_t>(B) * ROWS * d.Ls) ||
      own_alloc(e, &d.layer32, static_cast<size_t>(B) * ROWS * d.Ls) ||
      own_alloc(e, &d.knot, static_cast<size_t>(B) * d.nkmax) || own_alloc(e, &d.nknot, B) ||
      own_alloc(e, &d.seed, static_cast<size_t>(B) * d.nsmax) || own_alloc(e, &d.nseed, B) ||
      own_alloc(e, &d.nbr, nt) || own_alloc(e, &d.tflags, nt) ||
      own_alloc(e, &d.tr_model, nt) || own_alloc(e, &d.tr_stride, nt) || own_alloc(e, &d.tr_modes, nt) ||
      own_alloc(e, &d.tr_period, nt) || own_alloc(e, &d.tr_out, nt) ||
      own_alloc(e, &d.slot, nt * d.KB * SLOT) ||
      own_alloc(e, &d.trace_list, nt) || own_alloc(e, &d.repair_list, nt) ||
      own_alloc(e, &d.refine_list, 2 * nt * d.KB) ||
      own_alloc(e, &d.group_list, nt * nm) || own_alloc(e, &d.ctr, C_COUNT) ||
      own_alloc(e, &d.gwin, nt * nm * 2) ||
      own_alloc(e, &e->d_stats, static_cast<size_t>(MD200_STAT_COUNT) * md200_engine::MAX_CHUNKS))
    return 1;
  // host-path device buffers
  if (own_alloc(e, &e->in_h, static_cast<size_t>(B) * L) ||
      own_alloc(e, &e->in_vp, static_cast<size_t>(B) * L) ||
      own_alloc(e, &e->in_vs, static_cast<size_t>(B) * L) ||
      own_alloc(e, &e->in_rho, static_cast<size_t>(B) * L) || own_alloc(e, &e->in_per, T) ||
      own_alloc(e, &e->in_bounds, static_cast<size_t>(B) * 2) ||
      own_alloc(e, &e->out_vel, nt * nm) || own_alloc(e, &e->out_grp, nt * nm) ||
      own_alloc(e, &e->out_gflags, nt * nm) || own_alloc(e, &e->out_flags, nt) ||
      own_alloc(e, &e->out_pred, nt) || own_alloc(e, &e->out_levels, nt) ||
      own_alloc(e, &e->out_counts, nt) || own_alloc(e, &e->out_cflags, nt))
    return 1;
  // roots and counts of continuity suspects before their FP64 re-scan
  if (d.fp32 && e->o.continuity_check &&
      (own_alloc(e, &d.cold, nt * nm) || own_alloc(e, &d.ccount, nt)))
    return 1;
  // split FP32 scan: active lists, per-trace state, per-sample buffers
  if (d.fp32) {
    d.sp_cap = static_cast<int>(std::min<size_t>(nt, SPLIT_ACTIVE_MAX));
    const size_t ns = static_cast<size_t>(d.sp_cap) * SPLIT_SAMPLES;
    if (own_alloc(e, &d.sp_act[0], d.sp_cap) || own_alloc(e, &d.sp_act[1], d.sp_cap) ||
        own_alloc(e, &d.sp_state, nt) || own_alloc(e, &d.sp_s, ns) || own_alloc(e, &d.sp_tr, d.sp_cap) ||
        own_alloc(e, &d.sp_kf, nt) ||
        own_alloc(e, &d.sp_redo, ns) || own_alloc(e, &d.sp_zoom, d.sp_cap) ||
        own_alloc(e, &d.sp_zarg, static_cast<size_t>(d.sp_cap) * 8))
      return 1;
  }
  // anchor continuation: plan, anchor slopes and safety, target and root lists
  if (e->o.continuation &&
      (own_alloc(e, &d.crole, nt) || own_alloc(e, &d.cleft, nt) || own_alloc(e, &d.cright, nt) ||
       own_alloc(e, &d.cslope, nt * d.KB) || own_alloc(e, &d.csafe, nt) || own_alloc(e, &d.cont_list, nt) ||
       own_alloc(e, &d.croot_list, nt * d.KB) || own_alloc(e, &d.ccode, nt * d.KB)))
    return 1;
  e->pinned_bytes = sizeof(double) * (4 * static_cast<size_t>(B) * L + T + 2 * static_cast<size_t>(B)) +
                    nt * nm * (2 * sizeof(double) + sizeof(unsigned)) + nt * 4 * sizeof(int) + nt +
                    md200_engine::MAX_CHUNKS * MD200_STAT_COUNT * sizeof(unsigned long long) +
                    2 * sizeof(double) * B + 64;
  MD200_CK(cudaMallocHost(reinterpret_cast<void **>(&e->pinned), e->pinned_bytes));

  // launch shapes
  int sms = 148;
  MD200_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, e->device));
  e->scan_warps = e->o.warps_per_block > 0 ? std::min(4, e->o.warps_per_block) : 4;
  e->scan_smem64 = scan_smem(e->scan_warps, d.Ls, sizeof(double));
  e->scan_smem32 = scan_smem(e->scan_warps, d.Ls, sizeof(float));
  for (auto fn : {scan<double, 0>, scan<double, 1>})
    MD200_CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(std::max<size_t>(e->scan_smem64, 1024))));
  for (auto fn : {scan<float, 0>, scan<float, 1>})
    MD200_CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(std::max<size_t>(e->scan_smem32, 1024))));
  int occ64 = 0, occ32 = 0;
  MD200_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ64, scan<double, 0>, 32 * e->scan_warps,
                                                         e->scan_smem64));
  MD200_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ32, scan<float, 0>, 32 * e->scan_warps,
                                                         e->scan_smem32));
  if (e->o.blocks_per_sm > 0) {
    occ64 = std::min(occ64, e->o.blocks_per_sm);
    occ32 = std::min(occ32, e->o.blocks_per_sm);
  }
  e->scan_blocks64 = sms * std::max(1, occ64);
  e->scan_blocks32 = sms * std::max(1, occ32);
  e->list_blocks = sms * 8;
  const int sort_n = std::max(d.nlog + 1 + 2 * L, d.nsmax);
  int cap2 = 1;
  while (cap2 < sort_n) cap2 <<= 1;
  e->sortcap = cap2;
  e->prep_warps = 4;
  e->prep_smem = static_cast<size_t>(e->prep_warps) * cap2 * (sizeof(double) + sizeof(int));
  for (auto &x : e->ev) MD200_CK(cudaEventCreate(&x));
  for (auto &x : e->chunk_ev) MD200_CK(cudaEventCreateWithFlags(&x, cudaEventDisableTiming));
  for (auto &x : e->solved_ev) MD200_CK(cudaEventCreateWithFlags(&x, cudaEventDisableTiming));
  if (d.fp32)
    for (auto &x : e->sp_ev) MD200_CK(cudaEventCreate(&x));
  MD200_CK(cudaFuncSetAttribute(prep_models, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(std::max<size_t>(e->prep_smem, 1024))));
  return 0;
}

// Lazily allocated engine-owned buffer.
template <class T>
int lazy_alloc(md200_engine *e, T **p, size_t count) {
  if (*p) return 0;
  return own_alloc(e, p, count);
}

int validate_geometry(md200_engine *e, int models) {
  if (!e) return fail("modisp_b200: null engine");
  if (models < 1 || models > e->cap)
    return fail("modisp_b200: model count " + std::to_string(models) + " outside 1.." +
                std::to_string(e->cap));
  return 0;
}

// Ragged batches: traces in CSR order of the models (see Dev); uniform batches
// pass ntraces = 0 and no descriptor.
struct Ragged {
  int ntraces = 0;
  const int *offsets = nullptr, *modes = nullptr;
  const long long *outbase = nullptr;
};

// Rounds of the split FP32 scan for a run of nt traces over an active set of
// cap traces: enough for every trace of a typical run to finish (a trace takes
// a round per SPLIT_SAMPLES samples, most take two or three); traces still
// unfinished after them are handed to the fused kernel.
int split_rounds(int nt, int cap) {
  const int waves = (nt + cap - 1) / cap;
  return std::min(md200_engine::MAX_SPLIT_ROUNDS, 3 * waves + 6);
}

// The split FP32 scan's launches (split_scan.cuh): `rounds` rounds, then the
// fused kernel for the traces still unfinished (resumed from their state) and
// for any the rounds never took from the trace list.  Returns the launch count,
// or -1 when an event could not be recorded.
template <int WAVE>
int split_scan(md200_engine *e, const Dev &d, int rounds, cudaStream_t s) {
  const int sms = e->list_blocks / 8;
  const int cap = d.sp_cap;
  const int fill_blocks = std::max(1, std::min((cap + 255) / 256, sms * 8));
  const int pos_blocks = std::max(1, std::min((cap + 3) / 4, sms * 16));
  const int eval_blocks = sms * 16;
  const int book_blocks = std::max(1, std::min((cap + 127) / 128, sms * 8));
  int nl = 0;
  for (int r = 0; r < rounds; ++r) {
    const int p = r & 1;
    split_feed_count<<<1, 1, 0, s>>>(d, p);
    split_feed_fill<<<fill_blocks, 256, 0, s>>>(d, p);
    split_positions<<<pos_blocks, 128, 0, s>>>(d, p);
    if (!e->capturing && cudaEventRecord(e->sp_ev[2 * r], s) != cudaSuccess) return -1;
#if MD200_SPLIT_PAIR
    if (WAVE == 0)
      split_eval32_pair<<<sms * MD200_SPLIT_PAIR_GRID, 128, 0, s>>>(d, p);
    else
#endif
      split_eval32<WAVE><<<eval_blocks, 128, 0, s>>>(d, p);
    if (!e->capturing && cudaEventRecord(e->sp_ev[2 * r + 1], s) != cudaSuccess) return -1;
    split_redo<WAVE><<<sms * 8, 128, 0, s>>>(d, p);
    split_book<WAVE><<<book_blocks, 128, 0, s>>>(d, p);
    split_zoom<WAVE><<<sms * 4, 128, 0, s>>>(d, p);
    nl += 7;
  }
  e->sp_timed = e->capturing ? 0 : rounds;
  const int pf = rounds & 1;
  const dim3 grid(e->scan_blocks32), block(32 * e->scan_warps);
  scan<float, WAVE><<<grid, block, e->scan_smem32, s>>>(d, d.sp_act[pf], C_SP_RESUME, C_SP_ACT0 + pf, 1);
  scan<float, WAVE><<<grid, block, e->scan_smem32, s>>>(d, d.trace_list, C_SP_FEED, C_NTRACE, 0);
  return nl + 2;
}

int enqueue(md200_engine *e, const double *h, const double *vp, const double *vs, const double *rho,
            int B, const double *periods, const double *bounds, double tol, double accept, int wave,
            double *vel, unsigned *flags, int *levels, int *counts, double *grp, unsigned *gflags,
            unsigned *pred, unsigned char *cflags, double *bounds_out, unsigned long long *stats, cudaStream_t s,
            const Ragged &rg = Ragged()) {
  if (!(tol > 0.) || !(tol < 1.)) return fail("modisp_b200: c_tol_rel must lie in (0, 1)");
  if (wave != 0 && wave != 1) return fail("modisp_b200: wave must be 0 (Rayleigh) or 1 (Love)");
  if (e->d.group && (!grp || !gflags))
    return fail("modisp_b200: group-velocity engine needs group output arrays");
  MD200_CK(cudaSetDevice(e->device));
  Dev d = e->d;
  d.B = B;
  d.n_traces = rg.offsets ? rg.ntraces : B * e->T;
  d.ragged = rg.offsets ? 1 : 0;
  d.r_offsets = rg.offsets;
  d.r_modes = rg.modes;
  d.r_outbase = rg.outbase;
  d.wave = wave;
  d.tol = tol;
  d.accept = accept;
  d.h = h;
  d.vp = vp;
  d.vs = vs;
  d.rho = rho;
  d.periods = periods;
  d.bounds_in = bounds;
  d.vel = vel;
  d.oflags = flags;
  d.olevels = levels;
  d.ocounts = counts;
  d.grp = grp;
  d.gflags = gflags;
  d.stats = stats;
  d.pred = pred;
  const bool screen = d.fp32 && e->o.continuity_check;
  const bool cont = d.crole != nullptr;  // anchor continuation, each model over its own periods
  d.cflags = screen ? cflags : nullptr;
  if (!d.cflags) d.cold = nullptr, d.ccount = nullptr;
  d.bounds_out = bounds_out;
  const int nt = d.n_traces;
  int nl = 0;  // kernels launched by this run
  MD200_CK(cudaMemsetAsync(d.ctr, 0, sizeof(int) * C_COUNT, s));
  if (stats) MD200_CK(cudaMemsetAsync(stats, 0, sizeof(unsigned long long) * MD200_STAT_COUNT, s));
  // stage marks: 0 prep, 1 init, 2 scan, 3 refine, 4 repair collect, 5 repair scan,
  // 6 repair refine, 7 assemble, 8 group (empty stages record back-to-back events)
  // stage marks (not while a graph is being captured: the stage times are of
  // direct runs)
  auto mark = [&](int i) { return e->capturing ? cudaSuccess : cudaEventRecord(e->ev[i], s); };
  MD200_CK(mark(0));
  const int pw = e->prep_warps;
  prep_models<<<(B + pw - 1) / pw, 32 * pw, e->prep_smem, s>>>(d, e->sortcap, 0);
  ++nl;
  MD200_CK(cudaGetLastError());
  if (cont) {
    continuation_plan<<<(B + 127) / 128, 128, 0, s>>>(d, std::max(2, e->o.anchor_stride));
    ++nl;
    MD200_CK(cudaGetLastError());
  }
  MD200_CK(mark(1));
  init_traces<<<(nt + 255) / 256, 256, 0, s>>>(d);
  ++nl;
  MD200_CK(cudaGetLastError());
  if (d.fp32) {
    tail_values<<<(nt + 127) / 128, 128, 0, s>>>(d);
    ++nl;
    MD200_CK(cudaGetLastError());
  }
  MD200_CK(mark(2));
  // the split scan in auto mode: Rayleigh runs of SPLIT_MIN_TRACES traces or more
  // (the Love step is too cheap for the rounds to pay: measured slower)
  const bool split = d.fp32 && (e->o.scan_mode == 2 ||
                                (e->o.scan_mode == 0 && wave == 0 && nt >= SPLIT_MIN_TRACES));
  if (split) {
    const int rounds = split_rounds(nt, d.sp_cap);
    const int launched = wave == 0 ? split_scan<0>(e, d, rounds, s) : split_scan<1>(e, d, rounds, s);
    if (launched < 0) return fail("modisp_b200 CUDA: event record failed in the split scan");
    nl += launched;
  } else {
    e->sp_timed = 0;
    const dim3 grid(d.fp32 ? e->scan_blocks32 : e->scan_blocks64), block(32 * e->scan_warps);
    const size_t sm = d.fp32 ? e->scan_smem32 : e->scan_smem64;
    if (d.fp32 && wave == 0) scan<float, 0><<<grid, block, sm, s>>>(d, d.trace_list, C_SCAN_CURSOR, C_NTRACE);
    else if (d.fp32) scan<float, 1><<<grid, block, sm, s>>>(d, d.trace_list, C_SCAN_CURSOR, C_NTRACE);
    else if (wave == 0) scan<double, 0><<<grid, block, sm, s>>>(d, d.trace_list, C_SCAN_CURSOR, C_NTRACE);
    else scan<double, 1><<<grid, block, sm, s>>>(d, d.trace_list, C_SCAN_CURSOR, C_NTRACE);
    ++nl;
  }
  MD200_CK(cudaGetLastError());
  MD200_CK(mark(3));
  refine<<<e->list_blocks, 128, 0, s>>>(d);
  ++nl;
  MD200_CK(cudaGetLastError());
  MD200_CK(mark(4));
  if (d.fp32) {
    collect_repairs<<<(nt + 255) / 256, 256, 0, s>>>(d);
    ++nl;
    MD200_CK(mark(5));
    if (wave == 0)
      scan<double, 0><<<e->scan_blocks64, 32 * e->scan_warps, e->scan_smem64, s>>>(d, d.repair_list,
                                                                                 C_REPAIR_CURSOR, C_NREPAIR);
    else
      scan<double, 1><<<e->scan_blocks64, 32 * e->scan_warps, e->scan_smem64, s>>>(d, d.repair_list,
                                                                                 C_REPAIR_CURSOR, C_NREPAIR);
    ++nl;
    MD200_CK(mark(6));
    refine<<<e->list_blocks, 128, 0, s>>>(d);
    ++nl;
    MD200_CK(cudaGetLastError());
  } else {
    MD200_CK(mark(5));
    MD200_CK(mark(6));
  }
  MD200_CK(mark(7));
  assemble<<<(nt + 255) / 256, 256, 0, s>>>(d);
  ++nl;
  MD200_CK(cudaGetLastError());
  MD200_CK(mark(8));
  if (d.group) {
    group_velocity<<<e->list_blocks, 128, 0, s>>>(d);
    ++nl;
    MD200_CK(cudaGetLastError());
  }
  {
    // fallback: traces the first search could not finish, re-scanned in FP64 with
    // the larger point limit, refined, assembled and given group velocities again
    // (the lists are empty -- and the launches nearly free -- when there are none)
    MD200_CK(cudaMemsetAsync(d.ctr + C_REPAIR_CURSOR, 0, 2 * sizeof(int), s));
    collect_fallback<<<(nt + 255) / 256, 256, 0, s>>>(d);
    ++nl;
    Dev df = d;
    df.jmax = JMAX_FALLBACK;
    if (wave == 0)
      scan<double, 0><<<e->scan_blocks64, 32 * e->scan_warps, e->scan_smem64, s>>>(df, d.repair_list,
                                                                                 C_REPAIR_CURSOR, C_NREPAIR);
    else
      scan<double, 1><<<e->scan_blocks64, 32 * e->scan_warps, e->scan_smem64, s>>>(df, d.repair_list,
                                                                                 C_REPAIR_CURSOR, C_NREPAIR);
    ++nl;
    MD200_CK(cudaGetLastError());
    refine<<<e->list_blocks, 128, 0, s>>>(d);
    ++nl;
    assemble<<<(nt + 255) / 256, 256, 0, s>>>(d, d.repair_list, C_NREPAIR);
    ++nl;
    MD200_CK(cudaGetLastError());
    if (d.group) {
      group_velocity<<<e->list_blocks, 128, 0, s>>>(d);
      ++nl;
      MD200_CK(cudaGetLastError());
    }
  }
  if (cont) {
    // anchor continuation: the anchors are solved; predict, refine and audit the
    // targets, and send every doubtful one to the FP64 full search
    const size_t items = static_cast<size_t>(nt) * d.KB;
    MD200_CK(cudaMemsetAsync(d.ctr + C_REPAIR_CURSOR, 0, 2 * sizeof(int), s));
    anchor_slopes<<<static_cast<unsigned>((items + 255) / 256), 256, 0, s>>>(d);
    ++nl;
    continuation_predict<<<(nt + 255) / 256, 256, 0, s>>>(d);
    ++nl;
    continuation_root<<<static_cast<unsigned>((items + 127) / 128), 128, 0, s>>>(d);
    ++nl;
    continuation_audit<<<e->list_blocks, 128, 0, s>>>(d);
    ++nl;
    MD200_CK(cudaGetLastError());
    if (wave == 0)
      scan<double, 0><<<e->scan_blocks64, 32 * e->scan_warps, e->scan_smem64, s>>>(d, d.repair_list,
                                                                                 C_REPAIR_CURSOR, C_NREPAIR);
    else
      scan<double, 1><<<e->scan_blocks64, 32 * e->scan_warps, e->scan_smem64, s>>>(d, d.repair_list,
                                                                                 C_REPAIR_CURSOR, C_NREPAIR);
    ++nl;
    refine<<<e->list_blocks, 128, 0, s>>>(d);
    ++nl;
    assemble<<<(nt + 255) / 256, 256, 0, s>>>(d, d.cont_list, C_NTARGET);
    ++nl;
    MD200_CK(cudaGetLastError());
    if (d.group) {
      group_velocity<<<e->list_blocks, 128, 0, s>>>(d);
      ++nl;
      MD200_CK(cudaGetLastError());
    }
  }
  MD200_CK(mark(9));
  if (screen) {
    // FP64 continuity recheck: suspects of the continuity screen are re-scanned
    // in FP64, refined, assembled and given group velocities again
    MD200_CK(cudaMemsetAsync(d.ctr + C_REPAIR_CURSOR, 0, 2 * sizeof(int), s));
    continuity_screen<<<(nt + 255) / 256, 256, 0, s>>>(d);
    ++nl;
    MD200_CK(cudaGetLastError());
    if (wave == 0)
      scan<double, 0><<<e->scan_blocks64, 32 * e->scan_warps, e->scan_smem64, s>>>(d, d.repair_list,
                                                                                 C_REPAIR_CURSOR, C_NREPAIR);
    else
      scan<double, 1><<<e->scan_blocks64, 32 * e->scan_warps, e->scan_smem64, s>>>(d, d.repair_list,
                                                                                 C_REPAIR_CURSOR, C_NREPAIR);
    ++nl;
    MD200_CK(cudaGetLastError());
    refine<<<e->list_blocks, 128, 0, s>>>(d);
    ++nl;
    assemble<<<(nt + 255) / 256, 256, 0, s>>>(d, d.repair_list, C_NREPAIR);
    ++nl;
    MD200_CK(cudaGetLastError());
    if (d.group) {
      group_velocity<<<e->list_blocks, 128, 0, s>>>(d);
      ++nl;
      MD200_CK(cudaGetLastError());
    }
    if (d.cflags) {
      continuity_finish<<<(nt + 255) / 256, 256, 0, s>>>(d);
      ++nl;
      MD200_CK(cudaGetLastError());
    }
  } else if (cflags) {
    // no screen in this engine: every trace unscreened
    MD200_CK(cudaMemsetAsync(cflags, 0, static_cast<size_t>(nt), s));
  }
  MD200_CK(mark(10));
  if (!e->capturing) e->profiling = true;
  e->last_launches = nl;
  return 0;
}

// Jacobians of given roots: the models are prepared again (the layer tables are
// recomputed, not kept from the solve) and one thread per output cell runs the
// forward + adjoint sweeps.  Full Jacobians when grad is null, otherwise the
// weighted sum over cells into grad [4][B][Lmax].
int jacobian_enqueue(md200_engine *e, const double *h, const double *vp, const double *vs, const double *rho,
                     int B, const double *periods, int wave, const double *vel, const double *grp, double *jc,
                     double *ju, const double *wc, const double *wu, double *grad, cudaStream_t s) {
  if (wave != 0 && wave != 1) return fail("modisp_b200: wave must be 0 (Rayleigh) or 1 (Love)");
  if (e->L - 1 > JAC_MAX_STEPS)
    return fail("modisp_b200: Jacobians support models of at most " + std::to_string(JAC_MAX_STEPS + 1) +
                " rows");
  if (!vel) return fail("modisp_b200: Jacobians need the roots (velocity array)");
  MD200_CK(cudaSetDevice(e->device));
  Dev d = e->d;
  d.B = B;
  d.n_traces = B * e->T;
  d.wave = wave;
  d.h = h;
  d.vp = vp;
  d.vs = vs;
  d.rho = rho;
  d.periods = periods;
  d.bounds_in = nullptr;
  d.bounds_out = nullptr;
  d.stats = nullptr;
  d.pred = nullptr;
  MD200_CK(cudaMemsetAsync(d.ctr, 0, sizeof(int) * C_COUNT, s));
  const int pw = e->prep_warps;
  prep_models<<<(B + pw - 1) / pw, 32 * pw, e->prep_smem, s>>>(d, e->sortcap, 0);
  MD200_CK(cudaGetLastError());
  if (grad) MD200_CK(cudaMemsetAsync(grad, 0, sizeof(double) * 4 * static_cast<size_t>(B) * e->L, s));
  // One thread per output cell.  Most cells hold no root and their warps leave at
  // once; the block scheduler then keeps every SM on root-bearing warps.  A grid
  // capped at the resident blocks (each thread striding over many cells) left
  // threads with uneven shares and ran 3.2x slower.
  const long long cells = static_cast<long long>(B) * e->nmodes * e->T;
  const int blocks = static_cast<int>(std::min<long long>((cells + 127) / 128, 1LL << 30));
  if (wave == 0) root_jacobians<0><<<blocks, 128, 0, s>>>(d, vel, grp, jc, ju, wc, wu, grad, d.ctr + C_JFAIL);
  else root_jacobians<1><<<blocks, 128, 0, s>>>(d, vel, grp, jc, ju, wc, wu, grad, d.ctr + C_JFAIL);
  MD200_CK(cudaGetLastError());
  return 0;
}

}  // namespace

namespace {
// ---------------------------------------------------------------------------
// Static scratch for md200_group_roots_static: 2048 doubles (16 KiB), room for
// 7 x layers (prepared rows) + roots + modes (group velocities) + modes / 2 (flags)
// -- e.g. 256 layers with up to 100 roots and modes, or 100 layers with any count.
// Every GPU that loads this library holds it until the process exits.  In host
// code the symbol is only a handle: the device address comes from
// cudaGetSymbolAddress on the current device.
// ---------------------------------------------------------------------------
constexpr int STATIC_SCRATCH_DOUBLES = 2048;
static __device__ __align__(256) double g_group_scratch[STATIC_SCRATCH_DOUBLES];

// Device address of g_group_scratch on the current device.  Looked up on every
// call (a host-side table lookup, cheap next to the call's synchronous copies):
// a cached address would go stale if the caller reset the device between calls.
int static_scratch(double **address) {
  void *p = nullptr;
  MD200_CK(cudaGetSymbolAddress(&p, g_group_scratch));
  *address = static_cast<double *>(p);
  return 0;
}

// Sustained non-tensor FMA throughput (flop/s, an FMA counted as 2): 8 independent
// dependent-FMA chains per thread over every SM; the roofline denominator of the
// scan and refinement kernels.
template <class T>
__global__ void fma_chains(T *out, int iters, T a, T b) {
  T x[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) x[j] = static_cast<T>(threadIdx.x + j);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < 8; ++j) x[j] = fma(x[j], a, b);
  }
  T sum = 0;
#pragma unroll
  for (int j = 0; j < 8; ++j) sum += x[j];
  if (sum == static_cast<T>(-1.2345)) out[0] = sum;  // keeps the chains live
}

}  // namespace

extern "C" {

void md200_default_options(md200_options *o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->accuracy = 0;
  o->close_root_rtol = .005;
  o->shape = 1;
  o->sampling_rtol = 1e-3;
  o->refinement = 1;
  o->love_phase = 1;
  o->group_rtol = 1e-3;
  o->anchor_stride = 4;
  o->continuity_check = 1;
}

md200_engine *md200_create(int device, int capacity, int layers, int periods, int nmodes,
                           const md200_options *options) {
  if (capacity < 1 || layers < 1 || layers > 256 || periods < 1 || nmodes < 1 || nmodes > 256) {
    fail("modisp_b200: invalid engine geometry (capacity >= 1, 1 <= layers <= 256, periods >= 1, "
         "1 <= nmodes <= 256)");
    return nullptr;
  }
  md200_engine *e = new (std::nothrow) md200_engine();
  if (!e) {
    fail("modisp_b200: out of host memory");
    return nullptr;
  }
  e->device = device;
  e->cap = capacity;
  e->L = layers;
  e->T = periods;
  e->nmodes = nmodes;
  if (options) e->o = *options;
  else md200_default_options(&e->o);
  if (setup(e)) {
    const std::string msg = g_error;
    release(e);
    delete e;
    g_error = msg;
    return nullptr;
  }
  return e;
}

int md200_run_device(md200_engine *e, const double *h, const double *vp, const double *vs,
                     const double *rho, int models, const double *periods, const double *bounds,
                     double tol, double accept, int wave, double *velocity, unsigned *flags,
                     int *levels, int *counts, double *group, unsigned *group_flags,
                     unsigned *prediction_flags, uint8_t *continuity_flags, double *bounds_out,
                     unsigned long long *stats, void *stream) {
  if (validate_geometry(e, models)) return 1;
  if (!h || !vp || !vs || !rho || !periods || !velocity || !flags || !levels || !counts)
    return fail("modisp_b200: missing input or output array");
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : e->stream;
  return enqueue(e, h, vp, vs, rho, models, periods, bounds, tol, accept, wave, velocity, flags,
                 levels, counts, group, group_flags, prediction_flags, continuity_flags, bounds_out, stats, s);
}

int md200_run(md200_engine *e, const double *h, const double *vp, const double *vs,
              const double *rho, int models, const double *periods, const double *bounds,
              double tol, double accept, int wave, double *velocity, unsigned *flags, int *levels,
              int *counts, double *group, unsigned *group_flags, unsigned *prediction_flags,
              uint8_t *continuity_flags, double *bounds_out, unsigned long long *stats, int nstats) {
  try {
    if (validate_geometry(e, models)) return 1;
    if (!h || !vp || !vs || !rho || !periods || !velocity || !flags || !levels || !counts)
      return fail("modisp_b200: missing input or output array");
    if (e->d.group && (!group || !group_flags))
      return fail("modisp_b200: group-velocity engine needs group output arrays");
    MD200_CK(cudaSetDevice(e->device));
    // copies left in flight by a call that failed part-way write the staging buffer
    MD200_CK(cudaStreamSynchronize(e->copy_stream));
    const size_t B = models, L = e->L, T = e->T, nm = e->nmodes, nt = B * T;
    // stage inputs through pinned memory
    unsigned char *p = e->pinned;
    double *ph = reinterpret_cast<double *>(p);
    {
      std::vector<HostCopy> in = {{ph, h, sizeof(double) * B * L},
                                  {ph + B * L, vp, sizeof(double) * B * L},
                                  {ph + 2 * B * L, vs, sizeof(double) * B * L},
                                  {ph + 3 * B * L, rho, sizeof(double) * B * L},
                                  {ph + 4 * B * L, periods, sizeof(double) * T}};
      if (bounds) in.push_back({ph + 4 * B * L + T, bounds, sizeof(double) * 2 * B});
      parallel_copy(in);
    }
    cudaStream_t s = e->stream;
    MD200_CK(cudaMemcpyAsync(e->in_h, ph, sizeof(double) * B * L, cudaMemcpyHostToDevice, s));
    MD200_CK(cudaMemcpyAsync(e->in_vp, ph + B * L, sizeof(double) * B * L, cudaMemcpyHostToDevice, s));
    MD200_CK(cudaMemcpyAsync(e->in_vs, ph + 2 * B * L, sizeof(double) * B * L, cudaMemcpyHostToDevice, s));
    MD200_CK(cudaMemcpyAsync(e->in_rho, ph + 3 * B * L, sizeof(double) * B * L, cudaMemcpyHostToDevice, s));
    MD200_CK(cudaMemcpyAsync(e->in_per, ph + 4 * B * L, sizeof(double) * T, cudaMemcpyHostToDevice, s));
    if (bounds)
      MD200_CK(cudaMemcpyAsync(e->in_bounds, ph + 4 * B * L + T, sizeof(double) * 2 * B,
                               cudaMemcpyHostToDevice, s));
    const bool grp = e->d.group != 0;
    // Large batches run in chunks of models, every chunk's outputs copied back as
    // soon as it is solved, so the host copies (and first-touch page faults) of
    // chunk i overlap the solve of chunk i + 1.  Every trace is independent: the
    // results are those of one run.
    // (each chunk adds a scan tail, so only batches far larger than the GPU's
    // resident traces are split)
    const int nchunk = B >= 65536 ? 4 : 1;
    double *ov = reinterpret_cast<double *>(p);
    double *og = ov + nt * nm;
    unsigned *ogf = reinterpret_cast<unsigned *>(og + nt * nm);
    unsigned *ofl = ogf + nt * nm;
    int *olv = reinterpret_cast<int *>(ofl + nt);
    int *oct = olv + nt;
    unsigned *opr = reinterpret_cast<unsigned *>(oct + nt);
    unsigned long long *ost = reinterpret_cast<unsigned long long *>(
        (reinterpret_cast<uintptr_t>(opr + nt) + 7) & ~uintptr_t(7));
    double *obd = reinterpret_cast<double *>(ost + static_cast<size_t>(MD200_STAT_COUNT) * md200_engine::MAX_CHUNKS);
    unsigned char *ocf = reinterpret_cast<unsigned char *>(obd + 2 * B);
    // decreasing chunk sizes: the last chunk's copies are the only ones nothing
    // overlaps, so it is the smallest (the tenth of the batch)
    static const double edge[5] = {0., .4, .7, .9, 1.};
    auto chunk_begin = [&](int c) -> size_t {
      return nchunk == 1 ? B * c : (c >= nchunk ? B : static_cast<size_t>(B * edge[c]));
    };
    for (int c = 0; c < nchunk; ++c) {
      const size_t b0 = chunk_begin(c), nb = chunk_begin(c + 1) - b0;
      const size_t cm = b0 * nm * T, ct = b0 * T, cells = nb * nm * T, traces = nb * T;
      unsigned long long *cstats = e->d_stats + static_cast<size_t>(c) * MD200_STAT_COUNT;
      if (enqueue(e, e->in_h + b0 * L, e->in_vp + b0 * L, e->in_vs + b0 * L, e->in_rho + b0 * L,
                  static_cast<int>(nb), e->in_per, bounds ? e->in_bounds + 2 * b0 : nullptr, tol, accept, wave,
                  e->out_vel + cm, e->out_flags + ct, e->out_levels + ct, e->out_counts + ct,
                  grp ? e->out_grp + cm : nullptr, grp ? e->out_gflags + cm : nullptr,
                  prediction_flags ? e->out_pred + ct : nullptr, continuity_flags ? e->out_cflags + ct : nullptr,
                  e->in_bounds + 2 * b0, cstats, s))
        return 1;
      // this chunk's copies wait for its solve only; the next chunk is solved meanwhile
      cudaStream_t cs = e->copy_stream;
      MD200_CK(cudaEventRecord(e->solved_ev[c], s));
      MD200_CK(cudaStreamWaitEvent(cs, e->solved_ev[c], 0));
      MD200_CK(cudaMemcpyAsync(ov + cm, e->out_vel + cm, sizeof(double) * cells, cudaMemcpyDeviceToHost, cs));
      MD200_CK(cudaMemcpyAsync(ofl + ct, e->out_flags + ct, sizeof(unsigned) * traces, cudaMemcpyDeviceToHost, cs));
      MD200_CK(cudaMemcpyAsync(olv + ct, e->out_levels + ct, sizeof(int) * traces, cudaMemcpyDeviceToHost, cs));
      MD200_CK(cudaMemcpyAsync(oct + ct, e->out_counts + ct, sizeof(int) * traces, cudaMemcpyDeviceToHost, cs));
      if (grp) {
        MD200_CK(cudaMemcpyAsync(og + cm, e->out_grp + cm, sizeof(double) * cells, cudaMemcpyDeviceToHost, cs));
        MD200_CK(cudaMemcpyAsync(ogf + cm, e->out_gflags + cm, sizeof(unsigned) * cells, cudaMemcpyDeviceToHost, cs));
      }
      if (prediction_flags)
        MD200_CK(cudaMemcpyAsync(opr + ct, e->out_pred + ct, sizeof(unsigned) * traces, cudaMemcpyDeviceToHost, cs));
      if (continuity_flags)
        MD200_CK(cudaMemcpyAsync(ocf + ct, e->out_cflags + ct, traces, cudaMemcpyDeviceToHost, cs));
      // the prep stage wrote the windows it used over the (already consumed) input windows
      if (bounds_out)
        MD200_CK(cudaMemcpyAsync(obd + 2 * b0, e->in_bounds + 2 * b0, sizeof(double) * 2 * nb,
                                 cudaMemcpyDeviceToHost, cs));
      MD200_CK(cudaEventRecord(e->chunk_ev[c], cs));
    }
    MD200_CK(cudaMemcpyAsync(ost, e->d_stats, sizeof(unsigned long long) * MD200_STAT_COUNT * nchunk,
                             cudaMemcpyDeviceToHost, e->copy_stream));
    for (int c = 0; c < nchunk; ++c) {
      MD200_CK(cudaEventSynchronize(e->chunk_ev[c]));
      const size_t b0 = chunk_begin(c), nb = chunk_begin(c + 1) - b0;
      const size_t cm = b0 * nm * T, ct = b0 * T, cells = nb * nm * T, traces = nb * T;
      std::vector<HostCopy> out = {{velocity + cm, ov + cm, sizeof(double) * cells},
                                   {flags + ct, ofl + ct, sizeof(unsigned) * traces},
                                   {levels + ct, olv + ct, sizeof(int) * traces},
                                   {counts + ct, oct + ct, sizeof(int) * traces}};
      if (grp) {
        out.push_back({group + cm, og + cm, sizeof(double) * cells});
        out.push_back({group_flags + cm, ogf + cm, sizeof(unsigned) * cells});
      }
      if (prediction_flags) out.push_back({prediction_flags + ct, opr + ct, sizeof(unsigned) * traces});
      if (continuity_flags) out.push_back({continuity_flags + ct, ocf + ct, traces});
      if (bounds_out) out.push_back({bounds_out + 2 * b0, obd + 2 * b0, sizeof(double) * 2 * nb});
      parallel_copy(out, c + 1 == nchunk ? 16u : 8u);  // nothing left to overlap the last
    }
    MD200_CK(cudaStreamSynchronize(s));
    MD200_CK(cudaStreamSynchronize(e->copy_stream));
    if (stats && nstats > 0) {
      const int n = std::min(nstats, int(MD200_STAT_COUNT));
      for (int i = 0; i < n; ++i) {
        unsigned long long sum = 0;
        for (int c = 0; c < nchunk; ++c) sum += ost[static_cast<size_t>(c) * MD200_STAT_COUNT + i];
        stats[i] = sum;
      }
    }
    return 0;
  } catch (...) {
    return fail_exception();
  }
}

int md200_jacobian_device(md200_engine *e, const double *h, const double *vp, const double *vs,
                          const double *rho, int models, const double *periods, int wave,
                          const double *velocity, const double *group, double *jac_phase,
                          double *jac_group, void *stream) {
  if (validate_geometry(e, models)) return 1;
  if (!h || !vp || !vs || !rho || !periods || !jac_phase)
    return fail("modisp_b200: missing input or output array");
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : e->stream;
  return jacobian_enqueue(e, h, vp, vs, rho, models, periods, wave, velocity, group, jac_phase, jac_group,
                          nullptr, nullptr, nullptr, s);
}

int md200_vjp_device(md200_engine *e, const double *h, const double *vp, const double *vs,
                     const double *rho, int models, const double *periods, int wave,
                     const double *velocity, const double *group, const double *weight_phase,
                     const double *weight_group, double *grad, void *stream) {
  if (validate_geometry(e, models)) return 1;
  if (!h || !vp || !vs || !rho || !periods || !grad || (!weight_phase && !weight_group))
    return fail("modisp_b200: missing input or output array");
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : e->stream;
  return jacobian_enqueue(e, h, vp, vs, rho, models, periods, wave, velocity, group, nullptr, nullptr,
                          weight_phase, weight_group, grad, s);
}

namespace {
// Host-path staging shared by md200_jacobian and md200_vjp: inputs to the
// engine's device buffers, roots and group velocities to jac_w.
int stage_jacobian_inputs(md200_engine *e, const double *h, const double *vp, const double *vs,
                          const double *rho, int models, const double *periods, const double *velocity,
                          const double *group, const double *wc, const double *wu) {
  const size_t B = models, L = e->L, T = e->T, nm = e->nmodes, cells = B * T * nm;
  const size_t cap_cells = static_cast<size_t>(e->cap) * T * nm;
  if (lazy_alloc(e, &e->jac_w, 4 * cap_cells)) return 1;
  cudaStream_t s = e->stream;
  MD200_CK(cudaMemcpyAsync(e->in_h, h, sizeof(double) * B * L, cudaMemcpyHostToDevice, s));
  MD200_CK(cudaMemcpyAsync(e->in_vp, vp, sizeof(double) * B * L, cudaMemcpyHostToDevice, s));
  MD200_CK(cudaMemcpyAsync(e->in_vs, vs, sizeof(double) * B * L, cudaMemcpyHostToDevice, s));
  MD200_CK(cudaMemcpyAsync(e->in_rho, rho, sizeof(double) * B * L, cudaMemcpyHostToDevice, s));
  MD200_CK(cudaMemcpyAsync(e->in_per, periods, sizeof(double) * T, cudaMemcpyHostToDevice, s));
  MD200_CK(cudaMemcpyAsync(e->jac_w, velocity, sizeof(double) * cells, cudaMemcpyHostToDevice, s));
  if (group)
    MD200_CK(cudaMemcpyAsync(e->jac_w + cap_cells, group, sizeof(double) * cells, cudaMemcpyHostToDevice, s));
  if (wc) MD200_CK(cudaMemcpyAsync(e->jac_w + 2 * cap_cells, wc, sizeof(double) * cells, cudaMemcpyHostToDevice, s));
  if (wu) MD200_CK(cudaMemcpyAsync(e->jac_w + 3 * cap_cells, wu, sizeof(double) * cells, cudaMemcpyHostToDevice, s));
  return 0;
}
}  // namespace

int md200_jacobian(md200_engine *e, const double *h, const double *vp, const double *vs, const double *rho,
                   int models, const double *periods, int wave, const double *velocity, const double *group,
                   double *jac_phase, double *jac_group, int *failed) {
  if (validate_geometry(e, models)) return 1;
  if (!h || !vp || !vs || !rho || !periods || !velocity || !jac_phase)
    return fail("modisp_b200: missing input or output array");
  MD200_CK(cudaSetDevice(e->device));
  const size_t cap_cells = static_cast<size_t>(e->cap) * e->T * e->nmodes;
  const size_t n = static_cast<size_t>(models) * e->T * e->nmodes * 4 * e->L;
  if (lazy_alloc(e, &e->jac_c, cap_cells * 4 * e->L)) return 1;
  if (jac_group && lazy_alloc(e, &e->jac_u, cap_cells * 4 * e->L)) return 1;
  if (stage_jacobian_inputs(e, h, vp, vs, rho, models, periods, velocity, group, nullptr, nullptr)) return 1;
  if (jacobian_enqueue(e, e->in_h, e->in_vp, e->in_vs, e->in_rho, models, e->in_per, wave, e->jac_w,
                       group ? e->jac_w + cap_cells : nullptr, e->jac_c, jac_group ? e->jac_u : nullptr, nullptr,
                       nullptr, nullptr, e->stream))
    return 1;
  int nfail = 0;
  MD200_CK(cudaMemcpyAsync(&nfail, e->d.ctr + C_JFAIL, sizeof(int), cudaMemcpyDeviceToHost, e->stream));
  MD200_CK(cudaStreamSynchronize(e->stream));
  MD200_CK(cudaMemcpy(jac_phase, e->jac_c, sizeof(double) * n, cudaMemcpyDeviceToHost));
  if (jac_group) MD200_CK(cudaMemcpy(jac_group, e->jac_u, sizeof(double) * n, cudaMemcpyDeviceToHost));
  if (failed) *failed = nfail;
  return 0;
}

int md200_vjp(md200_engine *e, const double *h, const double *vp, const double *vs, const double *rho,
              int models, const double *periods, int wave, const double *velocity, const double *group,
              const double *weight_phase, const double *weight_group, double *grad) {
  if (validate_geometry(e, models)) return 1;
  if (!h || !vp || !vs || !rho || !periods || !velocity || !grad || (!weight_phase && !weight_group))
    return fail("modisp_b200: missing input or output array");
  MD200_CK(cudaSetDevice(e->device));
  const size_t cap_cells = static_cast<size_t>(e->cap) * e->T * e->nmodes;
  if (lazy_alloc(e, &e->jac_grad, 4 * static_cast<size_t>(e->cap) * e->L)) return 1;
  if (stage_jacobian_inputs(e, h, vp, vs, rho, models, periods, velocity, group, weight_phase, weight_group))
    return 1;
  if (jacobian_enqueue(e, e->in_h, e->in_vp, e->in_vs, e->in_rho, models, e->in_per, wave, e->jac_w,
                       group ? e->jac_w + cap_cells : nullptr, nullptr, nullptr,
                       weight_phase ? e->jac_w + 2 * cap_cells : nullptr,
                       weight_group ? e->jac_w + 3 * cap_cells : nullptr, e->jac_grad, e->stream))
    return 1;
  MD200_CK(cudaStreamSynchronize(e->stream));
  MD200_CK(cudaMemcpy(grad, e->jac_grad, sizeof(double) * 4 * static_cast<size_t>(models) * e->L,
                      cudaMemcpyDeviceToHost));
  return 0;
}

int md200_run_ragged_device(md200_engine *e, const double *h, const double *vp, const double *vs,
                            const double *rho, int models, int traces, const int *period_offsets,
                            const double *periods, const int *modes, const long long *out_offsets,
                            const double *bounds, double tol, double accept, int wave, double *velocity, unsigned *flags, int *levels, int *counts,
                            double *group, unsigned *group_flags, uint8_t *continuity_flags, unsigned long long *stats,
                            void *stream) {
  if (validate_geometry(e, models)) return 1;
  if (traces < 1 || static_cast<long long>(traces) > static_cast<long long>(e->cap) * e->T)
    return fail("modisp_b200: ragged trace count " + std::to_string(traces) + " outside 1.." +
                std::to_string(static_cast<long long>(e->cap) * e->T) + " (capacity x periods)");
  if (!h || !vp || !vs || !rho || !period_offsets || !periods || !modes || !out_offsets || !velocity || !flags ||
      !levels || !counts)
    return fail("modisp_b200: missing input or output array");
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : e->stream;
  Ragged rg;
  rg.ntraces = traces;
  rg.offsets = period_offsets;
  rg.modes = modes;
  rg.outbase = out_offsets;
  return enqueue(e, h, vp, vs, rho, models, periods, bounds, tol, accept, wave, velocity, flags, levels, counts,
                 group, group_flags, nullptr, continuity_flags, nullptr, stats, s, rg);
}

int md200_run_ragged(md200_engine *e, const double *h, const double *vp, const double *vs, const double *rho,
                     int models, const int *period_offsets, const double *periods, const int *modes,
                     const double *bounds, double tol, double accept, int wave, double *velocity, unsigned *flags, int *levels, int *counts,
                     double *group, unsigned *group_flags, uint8_t *continuity_flags, unsigned long long *stats,
                     int nstats) {
  try {
    if (validate_geometry(e, models)) return 1;
    if (!h || !vp || !vs || !rho || !period_offsets || !periods || !modes || !velocity || !flags || !levels ||
        !counts)
      return fail("modisp_b200: missing input or output array");
    if (e->d.group && (!group || !group_flags))
      return fail("modisp_b200: group-velocity engine needs group output arrays");
    // the CSR description, checked here (the device path trusts it)
    if (period_offsets[0] != 0) return fail("modisp_b200: period_offsets[0] must be 0");
    std::vector<long long> outbase(models);
    long long cells = 0;
    for (int b = 0; b < models; ++b) {
      const int nb = period_offsets[b + 1] - period_offsets[b];
      if (nb < 0) return fail("modisp_b200: period_offsets must be non-decreasing");
      if (modes[b] < 1 || modes[b] > e->nmodes)
        return fail("modisp_b200: modes[" + std::to_string(b) + "] = " + std::to_string(modes[b]) +
                    " outside 1.." + std::to_string(e->nmodes));
      outbase[b] = cells;
      cells += static_cast<long long>(modes[b]) * nb;
    }
    const int traces = period_offsets[models];
    if (traces < 1 || static_cast<long long>(traces) > static_cast<long long>(e->cap) * e->T)
      return fail("modisp_b200: ragged trace count " + std::to_string(traces) + " outside 1.." +
                  std::to_string(static_cast<long long>(e->cap) * e->T) + " (capacity x periods)");
    for (int t = 0; t < traces; ++t)
      if (!(periods[t] > 0.)) return fail("modisp_b200: periods must be positive");
    MD200_CK(cudaSetDevice(e->device));
    const size_t B = models, L = e->L, capt = static_cast<size_t>(e->cap) * e->T;
    if (lazy_alloc(e, &e->rg_offsets, static_cast<size_t>(e->cap) + 1) || lazy_alloc(e, &e->rg_modes, e->cap) ||
        lazy_alloc(e, &e->rg_outbase, e->cap) || lazy_alloc(e, &e->rg_periods, capt))
      return 1;
    cudaStream_t s = e->stream;
    MD200_CK(cudaStreamSynchronize(s));  // the staging buffers below are reused
    MD200_CK(cudaMemcpy(e->in_h, h, sizeof(double) * B * L, cudaMemcpyHostToDevice));
    MD200_CK(cudaMemcpy(e->in_vp, vp, sizeof(double) * B * L, cudaMemcpyHostToDevice));
    MD200_CK(cudaMemcpy(e->in_vs, vs, sizeof(double) * B * L, cudaMemcpyHostToDevice));
    MD200_CK(cudaMemcpy(e->in_rho, rho, sizeof(double) * B * L, cudaMemcpyHostToDevice));
    MD200_CK(cudaMemcpy(e->rg_offsets, period_offsets, sizeof(int) * (B + 1), cudaMemcpyHostToDevice));
    MD200_CK(cudaMemcpy(e->rg_modes, modes, sizeof(int) * B, cudaMemcpyHostToDevice));
    MD200_CK(cudaMemcpy(e->rg_outbase, outbase.data(), sizeof(long long) * B, cudaMemcpyHostToDevice));
    MD200_CK(cudaMemcpy(e->rg_periods, periods, sizeof(double) * traces, cudaMemcpyHostToDevice));
    if (bounds) MD200_CK(cudaMemcpy(e->in_bounds, bounds, sizeof(double) * 2 * B, cudaMemcpyHostToDevice));
    const bool grp = e->d.group != 0;
    Ragged rg;
    rg.ntraces = traces;
    rg.offsets = e->rg_offsets;
    rg.modes = e->rg_modes;
    rg.outbase = e->rg_outbase;
    if (enqueue(e, e->in_h, e->in_vp, e->in_vs, e->in_rho, models, e->rg_periods, bounds ? e->in_bounds : nullptr,
                tol, accept, wave,
                e->out_vel, e->out_flags, e->out_levels, e->out_counts, grp ? e->out_grp : nullptr,
                grp ? e->out_gflags : nullptr, nullptr, continuity_flags ? e->out_cflags : nullptr, nullptr,
                e->d_stats, s, rg))
      return 1;
    MD200_CK(cudaStreamSynchronize(s));
    MD200_CK(cudaMemcpy(velocity, e->out_vel, sizeof(double) * cells, cudaMemcpyDeviceToHost));
    MD200_CK(cudaMemcpy(flags, e->out_flags, sizeof(unsigned) * traces, cudaMemcpyDeviceToHost));
    MD200_CK(cudaMemcpy(levels, e->out_levels, sizeof(int) * traces, cudaMemcpyDeviceToHost));
    MD200_CK(cudaMemcpy(counts, e->out_counts, sizeof(int) * traces, cudaMemcpyDeviceToHost));
    if (grp) {
      MD200_CK(cudaMemcpy(group, e->out_grp, sizeof(double) * cells, cudaMemcpyDeviceToHost));
      MD200_CK(cudaMemcpy(group_flags, e->out_gflags, sizeof(unsigned) * cells, cudaMemcpyDeviceToHost));
    }
    if (continuity_flags) MD200_CK(cudaMemcpy(continuity_flags, e->out_cflags, traces, cudaMemcpyDeviceToHost));
    if (stats && nstats > 0)
      MD200_CK(cudaMemcpy(stats, e->d_stats, sizeof(unsigned long long) * std::min(nstats, int(MD200_STAT_COUNT)),
                          cudaMemcpyDeviceToHost));
    return 0;
  } catch (...) {
    return fail_exception();
  }
}

int md200_graph_begin(md200_engine *e) {
  if (!e) return fail("modisp_b200: null engine");
  if (e->capturing) return fail("modisp_b200: a graph capture is already open on this engine");
  MD200_CK(cudaSetDevice(e->device));
  MD200_CK(cudaStreamSynchronize(e->stream));
  MD200_CK(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
  e->capturing = true;
  return 0;
}

int md200_graph_end(md200_engine *e) {
  if (!e) return fail("modisp_b200: null engine");
  if (!e->capturing) return fail("modisp_b200: no graph capture is open on this engine");
  MD200_CK(cudaSetDevice(e->device));
  e->capturing = false;
  cudaGraph_t g = nullptr;
  MD200_CK(cudaStreamEndCapture(e->stream, &g));
  cudaGraphExec_t x = nullptr;
  const cudaError_t err = cudaGraphInstantiate(&x, g, 0);
  if (err != cudaSuccess) {
    cudaGraphDestroy(g);
    return fail(std::string("modisp_b200 CUDA: ") + cudaGetErrorString(err) + " (cudaGraphInstantiate)");
  }
  if (e->graph_exec) cudaGraphExecDestroy(e->graph_exec);
  if (e->graph) cudaGraphDestroy(e->graph);
  e->graph = g;
  e->graph_exec = x;
  return 0;
}

int md200_graph_launch(md200_engine *e, void *stream) {
  if (!e) return fail("modisp_b200: null engine");
  if (!e->graph_exec) return fail("modisp_b200: no captured graph on this engine");
  MD200_CK(cudaSetDevice(e->device));
  MD200_CK(cudaGraphLaunch(e->graph_exec, stream ? static_cast<cudaStream_t>(stream) : e->stream));
  return 0;
}

int md200_stage_times(md200_engine *e, double *ms, int n) {
  if (!e || !e->profiling) return fail("modisp_b200: no run to report");
  MD200_CK(cudaEventSynchronize(e->ev[md200_engine::NSTAGE]));
  for (int i = 0; i < n && i < md200_engine::NSTAGE; ++i) {
    float t = 0.f;
    MD200_CK(cudaEventElapsedTime(&t, e->ev[i], e->ev[i + 1]));
    ms[i] = t;
  }
  if (n > md200_engine::NSTAGE) {  // the split scan's evaluation launches
    double sum = 0.;
    for (int r = 0; r < e->sp_timed; ++r) {
      float t = 0.f;
      MD200_CK(cudaEventElapsedTime(&t, e->sp_ev[2 * r], e->sp_ev[2 * r + 1]));
      sum += t;
    }
    ms[md200_engine::NSTAGE] = sum;
  }
  return 0;
}

int md200_kernel_launches(md200_engine *e) {
  if (!e) return -1;
  if (e->last_launches >= 0) return e->last_launches;  // counted by the last run
  // before any run: the launches of a run without continuity flags requested
  const int check = e->d.fp32 && e->o.continuity_check ? 4 + (e->d.group ? 1 : 0) : 0;
  const int fallback = 4 + (e->d.group ? 1 : 0);
  return 6 + (e->d.fp32 ? 4 : 0) - (e->d.group ? 0 : 1) + fallback + check;
}

void md200_destroy(md200_engine *e) {
  if (!e) return;
  release(e);
  delete e;
}

const char *md200_last_error(void) { return g_error.c_str(); }

int md200_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

int md200_available(int device) {
  const int n = md200_device_count();
  if (device < 0 || device >= n) return 0;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return 0;
  return prop.major == 10 ? 1 : 0;
}

int md200_set_device(int device) {
  MD200_CK(cudaSetDevice(device));
  MD200_CK(cudaFree(nullptr));
  return 0;
}

int md200_memory_info(size_t *free_bytes, size_t *total_bytes) {
  MD200_CK(cudaMemGetInfo(free_bytes, total_bytes));
  return 0;
}

int md200_device_name(int device, char *name, int length) {
  cudaDeviceProp prop;
  MD200_CK(cudaGetDeviceProperties(&prop, device));
  if (name && length > 0) {
    std::snprintf(name, static_cast<size_t>(length), "%s", prop.name);
  }
  return 0;
}

int md200_kernel_report(int layers, int single_precision, char *json, int length) {
  struct Entry {
    const char *name;
    const void *fn;
  };
  const Entry entries[] = {
      {"prep_models", reinterpret_cast<const void *>(prep_models)},
      {"scan_fp64", reinterpret_cast<const void *>(scan<double, 0>)},
      {"scan_fp32", reinterpret_cast<const void *>(scan<float, 0>)},
      {"scan_fp64_love", reinterpret_cast<const void *>(scan<double, 1>)},
      {"scan_fp32_love", reinterpret_cast<const void *>(scan<float, 1>)},
      {"refine", reinterpret_cast<const void *>(refine)},
      {"assemble", reinterpret_cast<const void *>(assemble)},
      {"group_velocity", reinterpret_cast<const void *>(group_velocity)},
  };
  std::string out = "{\"search_kernel\": \"" + std::string(single_precision ? "scan_fp32" : "scan_fp64") +
                    "\", \"layers\": " + std::to_string(layers) + ", \"kernels\": {";
  bool first = true;
  for (const auto &en : entries) {
    cudaFuncAttributes a;
    if (cudaFuncGetAttributes(&a, en.fn) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    const int Ls = (layers + 3) & ~3;
    size_t dyn = 0;
    if (std::strncmp(en.name, "scan", 4) == 0)
      dyn = scan_smem(4, Ls, std::strcmp(en.name, "scan_fp32") == 0 ? sizeof(float) : sizeof(double));
    int blocks = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, en.fn, 128, dyn);
    cudaGetLastError();
    char buf[512];
    std::snprintf(buf, sizeof buf,
                  "%s\"%s\": {\"registers\": %d, \"local_bytes\": %zu, \"static_shared_bytes\": %zu, "
                  "\"dynamic_shared_bytes\": %zu, \"max_threads\": %d, \"blocks_per_sm_at_128\": %d}",
                  first ? "" : ", ", en.name, a.numRegs, a.localSizeBytes, a.sharedSizeBytes, dyn,
                  a.maxThreadsPerBlock, blocks);
    out += buf;
    first = false;
  }
  out += "}}";
  if (!json || length <= 0) return fail("modisp_b200: no output buffer");
  std::snprintf(json, static_cast<size_t>(length), "%s", out.c_str());
  return static_cast<int>(out.size()) < length ? 0 : fail("modisp_b200: report truncated");
}

int md200_group_roots(const double *h, const double *vp, const double *vs, const double *rho,
                      int layers, int wave, double period, const double *roots, int known,
                      int modes, double close_rtol, double *group, unsigned *group_flags) {
  try {
    if (layers < 1 || layers > 256 || modes < 1 || modes > 256 || known < 0 || known > 256 ||
        !(period > 0.))
      return fail("modisp_b200: invalid review trace");
    const int L = layers;
    std::vector<double> tab(static_cast<size_t>(EVAL_ROWS) * L + known + 1, 0.);
    for (int j = 0; j < L; ++j) {
      const double s = vs[j];
      tab[j] = j == L - 1 ? 0. : h[j];
      tab[L + j] = 1. / vp[j];
      tab[2 * L + j] = s > 0. ? 1. / s : 0.;
      tab[3 * L + j] = s * s;
      tab[4 * L + j] = rho[j];
      tab[5 * L + j] = 1. / rho[j];
      tab[6 * L + j] = s > 0. ? 1. / (rho[j] * s * s) : 0.;
    }
    for (int j = 0; j < known; ++j) tab[static_cast<size_t>(EVAL_ROWS) * L + j] = roots[j];
    double *dtab = nullptr, *dgrp = nullptr;
    unsigned *dfl = nullptr;
    MD200_CK(cudaMalloc(&dtab, sizeof(double) * tab.size()));
    cudaError_t err = cudaMalloc(&dgrp, sizeof(double) * modes);
    if (err == cudaSuccess) err = cudaMalloc(&dfl, sizeof(unsigned) * modes);
    if (err == cudaSuccess)
      err = cudaMemcpy(dtab, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice);
    if (err == cudaSuccess) {
      group_roots<<<(modes + 31) / 32, 32>>>(dtab, L, vs[0] == 0. ? 1 : 0, wave, TWO_PI / period,
                                            dtab + static_cast<size_t>(EVAL_ROWS) * L, known, modes,
                                            close_rtol, dgrp, dfl);
      err = cudaGetLastError();
    }
    if (err == cudaSuccess) err = cudaMemcpy(group, dgrp, sizeof(double) * modes, cudaMemcpyDeviceToHost);
    if (err == cudaSuccess)
      err = cudaMemcpy(group_flags, dfl, sizeof(unsigned) * modes, cudaMemcpyDeviceToHost);
    cudaFree(dtab);
    cudaFree(dgrp);
    cudaFree(dfl);
    if (err != cudaSuccess) return fail(std::string("modisp_b200 CUDA: ") + cudaGetErrorString(err));
    return 0;
  } catch (...) {
    return fail_exception();
  }
}

// ---------------------------------------------------------------------------
// Cross-period mode-reliability checks (python/modisp/reliability.py:49-145)
// ---------------------------------------------------------------------------
namespace {

// ln(b / a) for a <= b, through log1p for small gaps (reliability.py:7-9)
double log_gap(double a, double b) { return b - a < a ? std::log1p((b - a) / a) : std::log(b) - std::log(a); }

// Every index the kernel will follow must lie inside the arrays.
bool plan_ok(const md200_period_plan *plan, const int32_t *order, int T) {
  for (int t = 0; t < T; ++t) {
    const md200_period_plan &p = plan[t];
    if (order[t] < 0 || order[t] >= T) return false;
    if (!(p.kind & MD200_PLAN_FIRST) && (p.prev < 0 || p.prev >= T)) return false;
    if ((p.kind & MD200_PLAN_PREDICT) && (p.older < 0 || p.older >= T || !std::isfinite(p.ratio))) return false;
    if (p.dup_begin < 0 || p.dup_end < p.dup_begin || p.dup_end > T) return false;
  }
  return true;
}

int reliability_args(ReliabilityArgs &r, int B, int K, int T, const md200_period_plan *plan, const int32_t *order,
                     double close_rtol, double max_step, double pred_rtol) {
  if (B < 1 || K < 1 || T < 1) return fail("modisp_b200: expected velocity [B,K,T] with B, K, T >= 1");
  if (!plan || !order || !plan_ok(plan, order, T)) return fail("modisp_b200: invalid period plan");
  if (!(close_rtol > 0.) || !(max_step > 0.) || !(pred_rtol > 0.) || !std::isfinite(close_rtol) ||
      !std::isfinite(max_step) || !std::isfinite(pred_rtol))
    return fail("modisp_b200: tolerances must be finite and positive");
  r.B = B;
  r.K = K;
  r.T = T;
  r.close_rtol = close_rtol;
  r.max_step = max_step;
  r.pred_rtol = pred_rtol;
  return 0;
}

}  // namespace

int md200_reliability_plan(const double *periods, int T, double max_log_period_gap, md200_period_plan *plan,
                           int32_t *order) {
  try {
    if (T < 1) return fail("modisp_b200: no periods");
    for (int t = 0; t < T; ++t)
      if (!std::isfinite(periods[t]) || !(periods[t] > 0.)) return fail("modisp_b200: periods must be finite and positive");
    std::vector<int32_t> idx(T);
    for (int t = 0; t < T; ++t) idx[t] = t;
    std::stable_sort(idx.begin(), idx.end(), [&](int32_t a, int32_t b) { return periods[a] < periods[b]; });
    std::vector<int32_t> unique;
    int32_t group = -1;  // position in order of the current distinct period
    for (int q = 0; q < T; ++q) {
      const int32_t t = idx[q];
      order[q] = t;
      md200_period_plan &p = plan[t];
      p = md200_period_plan{-1, -1, 0, 0, 0, 0, 0.};
      if (unique.empty()) {
        p.kind = MD200_PLAN_FIRST;
      } else {
        const int32_t prev = unique.back();
        p.prev = prev;
        if (periods[t] == periods[prev]) {
          p.kind = MD200_PLAN_DUPLICATE;
          plan[prev].dup_end = q + 1;
          continue;
        }
        const double lg = log_gap(periods[prev], periods[t]);
        if (lg > max_log_period_gap) p.kind |= MD200_PLAN_GAP;
        if (unique.size() >= 2) {
          const int32_t older = unique[unique.size() - 2];
          const double den = log_gap(periods[older], periods[prev]);
          if (den <= max_log_period_gap && lg <= max_log_period_gap) {
            p.kind |= MD200_PLAN_PREDICT;
            p.older = older;
            p.ratio = lg / den;
          }
        }
      }
      group = q;
      p.dup_begin = p.dup_end = group + 1;
      unique.push_back(t);
    }
    return 0;
  } catch (...) {
    return fail_exception();
  }
}

int md200_mode_reliability_planned(const double *velocity, const uint32_t *trace_flags, const int64_t *root_count,
                                   int B, int K, int T, const md200_period_plan *plan, const int32_t *order,
                                   double close_root_rtol, double max_relative_step, double prediction_rtol,
                                   uint16_t *flags, uint8_t *assessed, void *stream) {
  if (B < 1 || K < 1 || T < 1 || !plan || !order)
    return fail("modisp_b200: expected velocity [B,K,T] with B, K, T >= 1 and a device plan");
  if (!(close_root_rtol > 0.) || !(max_relative_step > 0.) || !(prediction_rtol > 0.) ||
      !std::isfinite(close_root_rtol) || !std::isfinite(max_relative_step) || !std::isfinite(prediction_rtol))
    return fail("modisp_b200: tolerances must be finite and positive");
  ReliabilityArgs r{velocity, trace_flags, root_count, plan, order, B, K, T, close_root_rtol, max_relative_step,
                    prediction_rtol, flags, assessed};
  const size_t n = static_cast<size_t>(B) * T;
  const unsigned grid = static_cast<unsigned>((n + 255) / 256);
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : cudaStreamLegacy;
  switch (K) {  // the roots of a trace in registers, loops unrolled to the exact K
#define MD200_RELIABILITY_CASE(KK) \
  case KK: mode_reliability_small<KK><<<grid, 256, 0, s>>>(r); break;
    MD200_RELIABILITY_CASE(1) MD200_RELIABILITY_CASE(2) MD200_RELIABILITY_CASE(3) MD200_RELIABILITY_CASE(4)
    MD200_RELIABILITY_CASE(5) MD200_RELIABILITY_CASE(6) MD200_RELIABILITY_CASE(7) MD200_RELIABILITY_CASE(8)
    MD200_RELIABILITY_CASE(9) MD200_RELIABILITY_CASE(10) MD200_RELIABILITY_CASE(11) MD200_RELIABILITY_CASE(12)
#undef MD200_RELIABILITY_CASE
    default: mode_reliability<<<grid, 256, 0, s>>>(r);
  }
  MD200_CK(cudaGetLastError());
  return 0;
}

int md200_mode_reliability_device(const double *velocity, const uint32_t *trace_flags, const int64_t *root_count,
                                  int B, int K, int T, const md200_period_plan *plan, const int32_t *order,
                                  double close_root_rtol, double max_relative_step, double prediction_rtol,
                                  uint16_t *flags, uint8_t *assessed, void *stream) {
  ReliabilityArgs r{};
  if (reliability_args(r, B, K, T, plan, order, close_root_rtol, max_relative_step, prediction_rtol)) return 1;
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : cudaStreamLegacy;
  void *dplan = nullptr;
  const size_t plan_bytes = sizeof(md200_period_plan) * T, order_bytes = sizeof(int32_t) * T;
  MD200_CK(cudaMallocAsync(&dplan, plan_bytes + order_bytes, s));
  cudaError_t err = cudaMemcpyAsync(dplan, plan, plan_bytes, cudaMemcpyHostToDevice, s);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(static_cast<char *>(dplan) + plan_bytes, order, order_bytes, cudaMemcpyHostToDevice, s);
  int status = 0;
  if (err == cudaSuccess)
    status = md200_mode_reliability_planned(
        velocity, trace_flags, root_count, B, K, T, static_cast<const md200_period_plan *>(dplan),
        reinterpret_cast<const int32_t *>(static_cast<char *>(dplan) + plan_bytes), close_root_rtol,
        max_relative_step, prediction_rtol, flags, assessed, s);
  const cudaError_t err2 = cudaFreeAsync(dplan, s);
  if (status) return status;
  if (err == cudaSuccess) err = err2;
  if (err != cudaSuccess) return fail(std::string("modisp_b200 CUDA: ") + cudaGetErrorString(err));
  return 0;
}

int md200_mode_reliability(int device, const double *velocity, const uint32_t *trace_flags,
                           const int64_t *root_count, int B, int K, int T, const md200_period_plan *plan,
                           const int32_t *order, double close_root_rtol, double max_relative_step,
                           double prediction_rtol, uint16_t *flags, uint8_t *assessed) {
  ReliabilityArgs check{};
  if (reliability_args(check, B, K, T, plan, order, close_root_rtol, max_relative_step, prediction_rtol)) return 1;
  MD200_CK(cudaSetDevice(device));
  cudaStream_t s = nullptr;
  MD200_CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  const size_t cells = static_cast<size_t>(B) * K * T, traces = static_cast<size_t>(B) * T;
  double *dv = nullptr;
  uint32_t *dtf = nullptr;
  int64_t *dcnt = nullptr;
  uint16_t *dfl = nullptr;
  uint8_t *das = nullptr;
  cudaError_t err = cudaMallocAsync(&dv, sizeof(double) * cells, s);
  if (err == cudaSuccess && trace_flags) err = cudaMallocAsync(&dtf, sizeof(uint32_t) * traces, s);
  if (err == cudaSuccess && root_count) err = cudaMallocAsync(&dcnt, sizeof(int64_t) * traces, s);
  if (err == cudaSuccess) err = cudaMallocAsync(&dfl, sizeof(uint16_t) * cells, s);
  if (err == cudaSuccess) err = cudaMallocAsync(&das, sizeof(uint8_t) * cells, s);
  if (err == cudaSuccess) err = cudaMemcpyAsync(dv, velocity, sizeof(double) * cells, cudaMemcpyHostToDevice, s);
  if (err == cudaSuccess && dtf)
    err = cudaMemcpyAsync(dtf, trace_flags, sizeof(uint32_t) * traces, cudaMemcpyHostToDevice, s);
  if (err == cudaSuccess && dcnt)
    err = cudaMemcpyAsync(dcnt, root_count, sizeof(int64_t) * traces, cudaMemcpyHostToDevice, s);
  int status = 0;
  if (err == cudaSuccess)
    status = md200_mode_reliability_device(dv, dtf, dcnt, B, K, T, plan, order, close_root_rtol, max_relative_step,
                                           prediction_rtol, dfl, das, s);
  if (err == cudaSuccess && !status)
    err = cudaMemcpyAsync(flags, dfl, sizeof(uint16_t) * cells, cudaMemcpyDeviceToHost, s);
  if (err == cudaSuccess && !status)
    err = cudaMemcpyAsync(assessed, das, sizeof(uint8_t) * cells, cudaMemcpyDeviceToHost, s);
  for (void *ptr : {static_cast<void *>(dv), static_cast<void *>(dtf), static_cast<void *>(dcnt),
                    static_cast<void *>(dfl), static_cast<void *>(das)})
    if (ptr) cudaFreeAsync(ptr, s);
  const cudaError_t sync = cudaStreamSynchronize(s);
  cudaStreamDestroy(s);
  if (status) return status;
  if (err == cudaSuccess) err = sync;
  if (err != cudaSuccess) return fail(std::string("modisp_b200 CUDA: ") + cudaGetErrorString(err));
  return 0;
}

int md200_continuity_screen(int device, const double *periods, int T, const double *velocity, int B, int K,
                            const uint32_t *prediction, int single, int bilateral, uint8_t *flags, int *suspect) {
  try {
    if (T < 1 || B < 1 || K < 1 || !periods || !velocity || !flags)
      return fail("modisp_b200: continuity screening requires periods[T] and phases[B,K,T]");
    // period order as the reference takes it: ascending as given, else sorted
    // (cpp/cpu/continuity_screen.hpp:30-34; the same std::sort)
    std::vector<int> order(T);
    for (int j = 0; j < T; ++j) order[j] = j;
    if (bilateral && T > 2 && !std::is_sorted(periods, periods + T))
      std::sort(order.begin(), order.end(), [&](int i, int j) { return periods[i] < periods[j]; });
    MD200_CK(cudaSetDevice(device));
    const size_t traces = static_cast<size_t>(B) * T, cells = traces * K;
    const size_t bytes = sizeof(double) * (T + cells) + sizeof(int) * (T + 1) + sizeof(unsigned) * traces + traces;
    unsigned char *buf = nullptr;
    MD200_CK(cudaMalloc(&buf, bytes));
    double *dper = reinterpret_cast<double *>(buf), *dvel = dper + T;
    int *dord = reinterpret_cast<int *>(dvel + cells), *dsus = dord + T;
    unsigned *dpred = reinterpret_cast<unsigned *>(dsus + 1);
    unsigned char *dout = reinterpret_cast<unsigned char *>(dpred + traces);
    cudaError_t err = cudaMemcpy(dper, periods, sizeof(double) * T, cudaMemcpyHostToDevice);
    if (err == cudaSuccess) err = cudaMemcpy(dvel, velocity, sizeof(double) * cells, cudaMemcpyHostToDevice);
    if (err == cudaSuccess) err = cudaMemcpy(dord, order.data(), sizeof(int) * T, cudaMemcpyHostToDevice);
    if (err == cudaSuccess && prediction)
      err = cudaMemcpy(dpred, prediction, sizeof(unsigned) * traces, cudaMemcpyHostToDevice);
    if (err == cudaSuccess) err = cudaMemset(dsus, 0, sizeof(int));
    if (err == cudaSuccess) {
      continuity_screen_plain<<<static_cast<unsigned>((traces + 255) / 256), 256>>>(
          dper, dord, T, dvel, B, K, prediction ? dpred : nullptr, single, bilateral, dout, dsus);
      err = cudaGetLastError();
    }
    int sus = 0;
    if (err == cudaSuccess) err = cudaMemcpy(flags, dout, traces, cudaMemcpyDeviceToHost);
    if (err == cudaSuccess) err = cudaMemcpy(&sus, dsus, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(buf);
    if (err != cudaSuccess) return fail(std::string("modisp_b200 CUDA: ") + cudaGetErrorString(err));
    if (suspect) *suspect = sus;
    return 0;
  } catch (...) {
    return fail_exception();
  }
}

int md200_measure_peak(int device, int fp64, double *flops) {
  MD200_CK(cudaSetDevice(device));
  int sms = 0;
  MD200_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  void *out = nullptr;
  MD200_CK(cudaMalloc(&out, 64));
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  const int blocks = sms * 8, threads = 256, iters = fp64 ? 4096 : 16384;
  float best = 1e30f;
  for (int rep = 0; rep < 4; ++rep) {
    cudaEventRecord(a);
    if (fp64) fma_chains<double><<<blocks, threads>>>(static_cast<double *>(out), iters, 0.999999, 1e-7);
    else fma_chains<float><<<blocks, threads>>>(static_cast<float *>(out), iters, 0.999999f, 1e-7f);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float t = 0.f;
    cudaEventElapsedTime(&t, a, b);
    if (rep) best = std::min(best, t);  // the first launch warms up
  }
  const cudaError_t err = cudaGetLastError();
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(out);
  if (err != cudaSuccess) return fail(std::string("modisp_b200 CUDA: ") + cudaGetErrorString(err));
  *flops = 2.0 * 8.0 * iters * static_cast<double>(blocks) * threads / (best * 1e-3);
  return 0;
}

int md200_group_roots_static(const double *h, const double *vp, const double *vs, const double *rho,
                             int layers, int wave, double period, const double *roots, int known,
                             int modes, double close_rtol, double *group, unsigned *group_flags) {
  try {
    if (layers < 1 || layers > 256 || modes < 1 || modes > 256 || known < 0 || known > 256 ||
        !(period > 0.))
      return fail("modisp_b200: invalid review trace");
    const int L = layers;
    // table (7 rows x L) + roots + group velocities + flags (two per double)
    const int need = EVAL_ROWS * L + known + modes + (modes + 1) / 2;
    if (need > STATIC_SCRATCH_DOUBLES)
      return fail("modisp_b200: review trace needs " + std::to_string(need) +
                  " doubles of static scratch, the maximum is " + std::to_string(STATIC_SCRATCH_DOUBLES));
    double table[STATIC_SCRATCH_DOUBLES];  // host staging on the stack: no heap use either
    for (int j = 0; j < L; ++j) {
      const double sv = vs[j];
      table[j] = j == L - 1 ? 0. : h[j];
      table[L + j] = 1. / vp[j];
      table[2 * L + j] = sv > 0. ? 1. / sv : 0.;
      table[3 * L + j] = sv * sv;
      table[4 * L + j] = rho[j];
      table[5 * L + j] = 1. / rho[j];
      table[6 * L + j] = sv > 0. ? 1. / (rho[j] * sv * sv) : 0.;
    }
    for (int j = 0; j < known; ++j) table[EVAL_ROWS * L + j] = roots[j];
    double *scratch = nullptr;
    if (static_scratch(&scratch)) return 1;
    double *dtab = scratch, *dgrp = scratch + EVAL_ROWS * L + known;
    unsigned *dfl = reinterpret_cast<unsigned *>(dgrp + modes);
    // the table and roots are rewritten by every call, and the kernel writes every
    // output slot: nothing left by an earlier call is read
    MD200_CK(cudaMemcpy(dtab, table, sizeof(double) * (EVAL_ROWS * L + known), cudaMemcpyHostToDevice));
    group_roots<<<(modes + 31) / 32, 32>>>(dtab, L, vs[0] == 0. ? 1 : 0, wave, TWO_PI / period,
                                          dtab + EVAL_ROWS * L, known, modes, close_rtol, dgrp, dfl);
    MD200_CK(cudaGetLastError());
    MD200_CK(cudaMemcpy(group, dgrp, sizeof(double) * modes, cudaMemcpyDeviceToHost));
    MD200_CK(cudaMemcpy(group_flags, dfl, sizeof(unsigned) * modes, cudaMemcpyDeviceToHost));
    return 0;
  } catch (...) {
    return fail_exception();
  }
}


// ---------------------------------------------------------------------------
// Legacy uniform-grid path (the reference's search_strategy="uniform"): one
// object type for the reference's two stage states, md_cuda_state
// (cpp/cuda/coarse_scan.cu:63-300) and md_refine_state (cpp/cuda/refine.cu:48-400).
// A scan object holds the stage 1 rows, a refinement object the roots, flags and
// counters; both hold their models' tables.  All work runs on the legacy default
// stream, as the reference's does, so a refinement and the scan whose rows it
// reads, and the next scan that overwrites them, are ordered without events.
// ---------------------------------------------------------------------------
}  // extern "C"

struct md200_uniform {
  int B = 0, L = 0, nf = 0, nc = 0, K = 0;
  int alloc_nf = 0, alloc_nc = 0, alloc_K = 0;  // geometry of the allocated outputs
  bool models = false, ran = false;
  double cmin = 0., cmax = 0.;  // range of the last scan
  int sms = 148;
  double *in = nullptr, *layer64 = nullptr, *out = nullptr;
  float *layer32 = nullptr, *periods = nullptr, *rows = nullptr;
  int *mL = nullptr, *list = nullptr, *count = nullptr;
  unsigned *flags = nullptr;
  unsigned long long *stats = nullptr;
  UniformBracket *br = nullptr;
};

namespace {

UniformDev uniform_dev(const md200_uniform *u, const float *rows) {
  UniformDev d{};
  d.B = u->B;
  d.Lmax = u->L;
  d.Ls = u->L;
  d.nf = u->nf;
  d.nc = u->nc;
  d.K = u->K;
  const size_t n = static_cast<size_t>(u->B) * u->L;
  d.h = u->in;
  d.vp = u->in + n;
  d.vs = u->in + 2 * n;
  d.rho = u->in + 3 * n;
  d.layer64 = u->layer64;
  d.layer32 = u->layer32;
  d.mL = u->mL;
  d.periods = u->periods;
  d.rows = rows;
  d.out = u->out;
  d.flags = u->flags;
  d.stats = u->stats;
  d.br = u->br;
  d.list = u->list;
  d.count = u->count;
  return d;
}

void uniform_free_outputs(md200_uniform *u) {
  cudaFree(u->rows);
  cudaFree(u->out);
  cudaFree(u->flags);
  cudaFree(u->br);
  cudaFree(u->list);
  u->rows = nullptr;
  u->out = nullptr;
  u->flags = nullptr;
  u->br = nullptr;
  u->list = nullptr;
  u->alloc_nf = u->alloc_nc = u->alloc_K = 0;
}

// cpp/cuda/refine.cuh:38-45: halvings for |c1 - c2| <= tol at the grid minimum
int uniform_iters(double dc, double tol) {
  if (!(tol > 0.0) || !(dc > tol)) return 1;
  const int n = static_cast<int>(std::ceil(std::log2(dc / tol)));
  return n < 1 ? 1 : (n > 60 ? 60 : n);
}

std::string num(int x) { return std::to_string(x); }

int uniform_geometry(const md200_uniform *u, const char *who) {
  if (u->nf != u->alloc_nf || u->nc != u->alloc_nc)
    return fail(std::string(who) + ": geometry changed since allocation (allocated nf=" + num(u->alloc_nf) +
                " nc=" + num(u->alloc_nc) + ", now nf=" + num(u->nf) + " nc=" + num(u->nc) +
                "); call set_output() again");
  return 0;
}

// persistent grid: `per_sm` blocks per SM at most, fewer when there is less work
int uniform_blocks(const md200_uniform *u, long long units_per_block_work, long long work, int per_sm) {
  const long long need = (work + units_per_block_work - 1) / units_per_block_work;
  return static_cast<int>(std::max(1LL, std::min(need, static_cast<long long>(u->sms) * per_sm)));
}

}  // namespace

extern "C" {

md200_uniform *md200_uniform_create(int models, int layers) {
  try {
    if (models <= 0 || layers < 2) {
      fail("md200_uniform_create: bad shape B=" + num(models) + " L=" + num(layers) +
           " (L must be >= 2: layers plus half-space)");
      return nullptr;
    }
    auto *u = new md200_uniform;
    u->B = models;
    u->L = layers;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&u->sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t n = static_cast<size_t>(models) * layers;
    if (dalloc(&u->in, 4 * n) != cudaSuccess || dalloc(&u->layer64, ROWS * n) != cudaSuccess ||
        dalloc(&u->layer32, ROWS * n) != cudaSuccess || dalloc(&u->mL, models) != cudaSuccess ||
        dalloc(&u->stats, US_COUNT) != cudaSuccess || dalloc(&u->count, 1) != cudaSuccess) {
      const cudaError_t e = cudaGetLastError();
      md200_uniform_destroy(u);
      fail(std::string("md200_uniform_create: cudaMalloc (model arrays): ") + cudaGetErrorString(e));
      return nullptr;
    }
    return u;
  } catch (...) {
    fail_exception();
    return nullptr;
  }
}

void md200_uniform_destroy(md200_uniform *u) {
  if (!u) return;
  uniform_free_outputs(u);
  cudaFree(u->in);
  cudaFree(u->layer64);
  cudaFree(u->layer32);
  cudaFree(u->mL);
  cudaFree(u->periods);
  cudaFree(u->stats);
  cudaFree(u->count);
  delete u;
}

int md200_uniform_models(md200_uniform *u, const double *h, const double *vp, const double *vs,
                         const double *rho) {
  try {
    if (!u || !h || !vp || !vs || !rho) return fail("md200_uniform_models: null argument");
    const size_t n = static_cast<size_t>(u->B) * u->L;
    for (size_t i = 0; i < n; ++i)
      if (!(vs[i] > 0.) || !(vp[i] > 0.) || !(rho[i] > 0.))
        return fail("md200_uniform_models: the uniform path takes solid models (vp, vs, rho > 0 in every row)");
    const double *src[4] = {h, vp, vs, rho};
    for (int i = 0; i < 4; ++i)
      MD200_CK(cudaMemcpy(u->in + i * n, src[i], n * sizeof(double), cudaMemcpyHostToDevice));
    uniform_prep<<<(u->B + 3) / 4, 128>>>(uniform_dev(u, nullptr));
    MD200_CK(cudaGetLastError());
    u->models = true;
    return 0;
  } catch (...) {
    return fail_exception();
  }
}

int md200_uniform_periods(md200_uniform *u, int periods, const double *values) {
  try {
    if (!u || !values) return fail("md200_uniform_periods: null argument");
    if (periods <= 0) return fail("md200_uniform_periods: nf must be positive, got " + num(periods));
    // a different period count invalidates outputs sized against the old one
    if (periods != u->nf) uniform_free_outputs(u);
    cudaFree(u->periods);
    u->periods = nullptr;
    MD200_CK(dalloc(&u->periods, periods));
    std::vector<float> single(values, values + periods);  // the reference keeps periods in single precision
    MD200_CK(cudaMemcpy(u->periods, single.data(), sizeof(float) * periods, cudaMemcpyHostToDevice));
    u->nf = periods;
    return 0;
  } catch (...) {
    return fail_exception();
  }
}

int md200_uniform_grid(md200_uniform *u, int nc, int nmodes) {
  try {
    if (!u) return fail("md200_uniform_grid: null state");
    if (nmodes < 0) return fail("md200_uniform_grid: nmodes must be >= 0, got " + num(nmodes));
    if (nmodes == 0 && nc <= 0) return fail("md200_uniform_grid: nc must be positive, got " + num(nc));
    if (nmodes > 0 && nc < 2)
      return fail("md200_uniform_grid: need nc >= 2 and nmodes >= 1, got nc=" + num(nc) + " nmodes=" +
                  num(nmodes));
    if (u->nf <= 0)
      return fail("md200_uniform_grid: upload_periods() first -- the output size depends on the period count");
    const size_t rows = static_cast<size_t>(u->B) * u->nf;
    if (nmodes > 0 && rows * nmodes >= (1ull << 31))
      return fail("md200_uniform_grid: models x periods x modes must stay below 2^31");
    uniform_free_outputs(u);
    if (nmodes == 0) {
      MD200_CK(dalloc(&u->rows, rows * nc));
    } else {
      MD200_CK(dalloc(&u->out, rows * nmodes));
      MD200_CK(dalloc(&u->flags, rows));
      MD200_CK(dalloc(&u->br, rows * nmodes));
      MD200_CK(dalloc(&u->list, rows * nmodes));
      u->K = u->alloc_K = nmodes;
    }
    u->nc = u->alloc_nc = nc;
    u->alloc_nf = u->nf;
    return 0;
  } catch (...) {
    return fail_exception();
  }
}

int md200_uniform_scan(md200_uniform *u, double cmin, double cmax) {
  try {
    if (!u || !u->periods) return fail("md200_uniform_scan: periods not uploaded");
    if (!u->rows) return fail("md200_uniform_scan: output not allocated");
    if (!u->models) return fail("md200_uniform_scan: models not uploaded");
    if (uniform_geometry(u, "md200_uniform_scan")) return 1;
    const double dc = u->nc > 1 ? (cmax - cmin) / static_cast<double>(u->nc - 1) : 0.;
    const long long warps = static_cast<long long>(u->B) * u->nf * ((u->nc + 31) / 32);
    uniform_scan<<<uniform_blocks(u, 8, warps, 16), 256>>>(uniform_dev(u, nullptr), u->rows, cmin, dc);
    MD200_CK(cudaGetLastError());
    u->cmin = cmin;
    u->cmax = cmax;
    u->ran = true;
    return 0;
  } catch (...) {
    return fail_exception();
  }
}

int md200_uniform_rows(md200_uniform *u, float *rows) {
  try {
    if (!u || !rows) return fail("md200_uniform_rows: null argument");
    if (!u->rows) return fail("md200_uniform_rows: output not allocated");
    if (uniform_geometry(u, "md200_uniform_rows")) return 1;
    MD200_CK(cudaMemcpy(rows, u->rows, sizeof(float) * u->B * static_cast<size_t>(u->nf) * u->nc,
                        cudaMemcpyDeviceToHost));
    return 0;
  } catch (...) {
    return fail_exception();
  }
}

int md200_uniform_set_rows(md200_uniform *u, const float *rows, double cmin, double cmax) {
  try {
    if (!u || !rows) return fail("md200_uniform_set_rows: null argument");
    if (!u->rows) return fail("md200_uniform_set_rows: output not allocated");
    if (uniform_geometry(u, "md200_uniform_set_rows")) return 1;
    MD200_CK(cudaMemcpy(u->rows, rows, sizeof(float) * u->B * static_cast<size_t>(u->nf) * u->nc,
                        cudaMemcpyHostToDevice));
    u->cmin = cmin;
    u->cmax = cmax;
    u->ran = true;
    return 0;
  } catch (...) {
    return fail_exception();
  }
}

int md200_uniform_refine(md200_uniform *u, const md200_uniform *scan, double cmin, double cmax, double c_tol_rel,
                         double f_accept, int nmodes) {
  try {
    if (!u || !u->periods) return fail("md200_uniform_refine: periods not uploaded");
    if (!u->out || !u->flags) return fail("md200_uniform_refine: output not allocated");
    if (!u->models) return fail("md200_uniform_refine: models not uploaded");
    if (!scan || !scan->rows) return fail("md200_uniform_refine: null scan buffer");
    if (uniform_geometry(u, "md200_uniform_refine")) return 1;
    if (nmodes > u->alloc_K)
      return fail("md200_uniform_refine: nmodes=" + num(nmodes) + " exceeds the allocated " + num(u->alloc_K) +
                  "; call set_output(nc, nmodes) to resize");
    if (scan->B != u->B || scan->L != u->L || scan->nf != u->nf || scan->nc != u->nc)
      return fail("md200_uniform_refine: scan and refine geometries differ");
    if (!scan->ran) return fail("md200_uniform_refine: the scan has not been run");
    if (scan->cmin != cmin || scan->cmax != cmax) return fail("md200_uniform_refine: scan and refine ranges differ");
    if (nmodes > 0) u->K = nmodes;
    const double dc = u->nc > 1 ? (cmax - cmin) / static_cast<double>(u->nc - 1) : 0.;
    const int iters = uniform_iters(dc, c_tol_rel * cmin);
    const size_t rows = static_cast<size_t>(u->B) * u->nf;
    MD200_CK(cudaMemset(u->stats, 0, sizeof(unsigned long long) * US_COUNT));
    MD200_CK(cudaMemset(u->flags, 0, sizeof(unsigned) * rows));
    MD200_CK(cudaMemset(u->count, 0, sizeof(int)));
    const UniformDev d = uniform_dev(u, scan->rows);
    uniform_walk<<<uniform_blocks(u, 4, static_cast<long long>(rows), 16), 128>>>(d, cmin, dc);
    MD200_CK(cudaGetLastError());
    uniform_bisect<<<uniform_blocks(u, 128, static_cast<long long>(rows) * u->K, 8), 128>>>(d, cmin, dc, iters,
                                                                                           f_accept);
    MD200_CK(cudaGetLastError());
    u->ran = true;
    return 0;
  } catch (...) {
    return fail_exception();
  }
}

int md200_uniform_sync(void) {
  MD200_CK(cudaStreamSynchronize(nullptr));
  return 0;
}

int md200_uniform_velocity(md200_uniform *u, double *velocity) {
  try {
    if (!u || !velocity) return fail("md200_uniform_velocity: null argument");
    if (!u->out) return fail("md200_uniform_velocity: output not allocated");
    if (uniform_geometry(u, "md200_uniform_velocity")) return 1;
    MD200_CK(cudaMemcpy(velocity, u->out, sizeof(double) * u->B * static_cast<size_t>(u->nf) * u->K,
                        cudaMemcpyDeviceToHost));
    return 0;
  } catch (...) {
    return fail_exception();
  }
}

int md200_uniform_flags(md200_uniform *u, uint32_t *flags) {
  try {
    if (!u || !flags) return fail("md200_uniform_flags: null argument");
    if (!u->flags) return fail("md200_uniform_flags: no flags allocated -- call set_output() and run() first");
    MD200_CK(cudaMemcpy(flags, u->flags, sizeof(uint32_t) * u->B * static_cast<size_t>(u->nf),
                        cudaMemcpyDeviceToHost));
    return 0;
  } catch (...) {
    return fail_exception();
  }
}

int md200_uniform_stats(md200_uniform *u, uint64_t *stats, int n) {
  try {
    if (!u || !stats) return fail("md200_uniform_stats: null argument");
    if (n < US_COUNT)
      return fail("md200_uniform_stats: need room for " + num(US_COUNT) + " counters, got " + num(n));
    unsigned long long h[US_COUNT];
    MD200_CK(cudaMemcpy(h, u->stats, sizeof(h), cudaMemcpyDeviceToHost));
    for (int i = 0; i < US_COUNT; ++i) stats[i] = h[i];
    return 0;
  } catch (...) {
    return fail_exception();
  }
}

int md200_uniform_iterations(double dc, double c_tol_rel, double cmin) { return uniform_iters(dc, c_tol_rel * cmin); }

int md200_uniform_kernel_report(int stage, int layers, int block, char *text, int length) {
  try {
    if (!text || length <= 0) return fail("md200_uniform_kernel_report: null buffer");
    const void *fn = stage == 0 ? reinterpret_cast<const void *>(uniform_scan)
                                : reinterpret_cast<const void *>(uniform_bisect);
    const int threads = stage == 0 ? 256 : 128;
    cudaFuncAttributes a{};
    MD200_CK(cudaFuncGetAttributes(&a, fn));
    int blocks = 0;
    MD200_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, fn, threads, 0));
    int dev = 0, per_sm = 2048;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxThreadsPerMultiProcessor, dev);
    std::snprintf(text, length,
                  "kernel=%s regs=%d spill_bytes=%d smem_static=%zu smem_dynamic=0 block=%d "
                  "max_blocks_per_sm=%d threads_per_sm=%d occupancy=%.1f%% layers=%d requested_block=%d",
                  stage == 0 ? "uniform_scan" : "uniform_bisect", a.numRegs, static_cast<int>(a.localSizeBytes),
                  a.sharedSizeBytes, threads, blocks, blocks * threads, 100.0 * blocks * threads / per_sm, layers,
                  block);
    return 0;
  } catch (...) {
    return fail_exception();
  }
}

}  // extern "C"
