"""ctypes binding of the engine's C ABI (include/modisp_b200.h).

The library is loaded from ``modisp_b200/_lib``.  There is no fallback: if the
library is missing or cannot be loaded, every entry point raises
``BackendUnavailableError`` with the reason.
"""
from __future__ import annotations

import ctypes
import threading
from pathlib import Path

import numpy as np

LIBRARY = Path(__file__).resolve().parent / "_lib" / "libmodisp_b200.so"
ABI_VERSION = 3
STAT_NAMES = ("evaluations", "evaluations_fp32", "layer_steps", "layer_steps_fp32", "brackets",
              "trough_probes", "probe_pairs", "fp64_repair_traces", "unconverged", "group_roots",
              "roots", "traces", "dual_layer_steps", "continuation_accepted",
              "continuation_fallbacks", "continuity_rescans", "fallback_rescans", "continuation_anchors",
              "continuation_evaluations", "split_eval_layer_steps")
STAT_COUNT = 20


class BackendUnavailableError(RuntimeError):
    """The B200 engine cannot run here (library or GPU missing)."""


class Options(ctypes.Structure):
    _fields_ = [
        ("accuracy", ctypes.c_int),
        ("period_threshold", ctypes.c_double),
        ("close_root_rtol", ctypes.c_double),
        ("shape", ctypes.c_int),
        ("sampling_rtol", ctypes.c_double),
        ("secular", ctypes.c_int),
        ("refinement", ctypes.c_int),
        ("love_phase", ctypes.c_int),
        ("single_precision", ctypes.c_int),
        ("group_velocity", ctypes.c_int),
        ("group_rtol", ctypes.c_double),
        ("continuation", ctypes.c_int),
        ("anchor_stride", ctypes.c_int),
        ("scan_density", ctypes.c_double),
        ("log_points", ctypes.c_int),
        ("warps_per_block", ctypes.c_int),
        ("blocks_per_sm", ctypes.c_int),
        ("continuity_check", ctypes.c_int),
        ("scan_points", ctypes.c_longlong),
        ("scan_mode", ctypes.c_int),
    ]


_lib = None
_lock = threading.Lock()
_P = ctypes.c_void_p
_D = ctypes.c_double
_I = ctypes.c_int

EXPORTS = {
    "md200_default_options": (None, [ctypes.POINTER(Options)]),
    "md200_create": (_P, [_I, _I, _I, _I, _I, ctypes.POINTER(Options)]),
    "md200_run": (_I, [_P, _P, _P, _P, _P, _I, _P, _P, _D, _D, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _I]),
    "md200_run_device": (_I, [_P, _P, _P, _P, _P, _I, _P, _P, _D, _D, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P,
                              _P]),
    "md200_destroy": (None, [_P]),
    "md200_last_error": (ctypes.c_char_p, []),
    "md200_device_count": (_I, []),
    "md200_available": (_I, [_I]),
    "md200_set_device": (_I, [_I]),
    "md200_memory_info": (_I, [ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t)]),
    "md200_device_name": (_I, [_I, ctypes.c_char_p, _I]),
    "md200_kernel_report": (_I, [_I, _I, ctypes.c_char_p, _I]),
    "md200_group_roots": (_I, [_P, _P, _P, _P, _I, _I, _D, _P, _I, _I, _D, _P, _P]),
    "md200_group_roots_static": (_I, [_P, _P, _P, _P, _I, _I, _D, _P, _I, _I, _D, _P, _P]),
    "md200_stage_times": (_I, [_P, ctypes.POINTER(ctypes.c_double), _I]),
    "md200_kernel_launches": (_I, [_P]),
    "md200_measure_peak": (_I, [_I, _I, ctypes.POINTER(ctypes.c_double)]),
    "md200_continuity_screen": (_I, [_I, _P, _I, _P, _I, _I, _P, _I, _I, _P, ctypes.POINTER(_I)]),
    "md200_run_ragged": (_I, [_P, _P, _P, _P, _P, _I, _P, _P, _P, _P, _D, _D, _I, _P, _P, _P, _P, _P, _P, _P,
                              _P, _I]),
    "md200_run_ragged_device": (_I, [_P, _P, _P, _P, _P, _I, _I, _P, _P, _P, _P, _P, _D, _D, _I, _P, _P, _P, _P,
                                     _P, _P, _P, _P, _P]),
    "md200_graph_begin": (_I, [_P]),
    "md200_graph_end": (_I, [_P]),
    "md200_graph_launch": (_I, [_P, _P]),
    "md200_jacobian_device": (_I, [_P, _P, _P, _P, _P, _I, _P, _I, _P, _P, _P, _P, _P]),
    "md200_jacobian": (_I, [_P, _P, _P, _P, _P, _I, _P, _I, _P, _P, _P, _P, ctypes.POINTER(_I)]),
    "md200_vjp_device": (_I, [_P, _P, _P, _P, _P, _I, _P, _I, _P, _P, _P, _P, _P, _P]),
    "md200_vjp": (_I, [_P, _P, _P, _P, _P, _I, _P, _I, _P, _P, _P, _P, _P]),
    "md200_reliability_plan": (_I, [_P, _I, _D, _P, _P]),
    "md200_mode_reliability": (_I, [_I, _P, _P, _P, _I, _I, _I, _P, _P, _D, _D, _D, _P, _P]),
    "md200_mode_reliability_device": (_I, [_P, _P, _P, _I, _I, _I, _P, _P, _D, _D, _D, _P, _P, _P]),
    "md200_mode_reliability_planned": (_I, [_P, _P, _P, _I, _I, _I, _P, _P, _D, _D, _D, _P, _P, _P]),
    "md200_uniform_create": (_P, [_I, _I]),
    "md200_uniform_destroy": (None, [_P]),
    "md200_uniform_models": (_I, [_P, _P, _P, _P, _P]),
    "md200_uniform_periods": (_I, [_P, _I, _P]),
    "md200_uniform_grid": (_I, [_P, _I, _I]),
    "md200_uniform_scan": (_I, [_P, _D, _D]),
    "md200_uniform_rows": (_I, [_P, _P]),
    "md200_uniform_set_rows": (_I, [_P, _P, _D, _D]),
    "md200_uniform_refine": (_I, [_P, _P, _D, _D, _D, _D, _I]),
    "md200_uniform_sync": (_I, []),
    "md200_uniform_velocity": (_I, [_P, _P]),
    "md200_uniform_flags": (_I, [_P, _P]),
    "md200_uniform_stats": (_I, [_P, _P, _I]),
    "md200_uniform_iterations": (_I, [_D, _D, _D]),
    "md200_uniform_kernel_report": (_I, [_I, _I, _I, ctypes.c_char_p, _I]),
}
# counters of the legacy uniform path, in C ABI order (cpp/cuda/bindings.cpp:58-59)
UNIFORM_STAT_NAMES = ("brackets", "rejected_sign", "rejected_f", "troughs", "hidden_roots", "relocated")
# md200_period_plan (include/modisp_b200.h)
PERIOD_PLAN = np.dtype([("prev", np.int32), ("older", np.int32), ("kind", np.int32), ("dup_begin", np.int32),
                        ("dup_end", np.int32), ("reserved", np.int32), ("ratio", np.float64)])
PLAN_FIRST, PLAN_DUPLICATE, PLAN_GAP, PLAN_PREDICT = 1, 2, 4, 8
STAGES = ("prep", "trace_list", "scan", "refine", "repair_select", "repair_scan", "repair_refine",
          "assemble", "group_velocity", "continuity", "scan_eval")


def lib():
    """The loaded engine library (raises BackendUnavailableError if absent)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not LIBRARY.exists():
                raise BackendUnavailableError(
                    f"engine library {LIBRARY} is not built; run `python -m modisp_b200.build`")
            try:
                handle = ctypes.CDLL(str(LIBRARY))
            except OSError as exc:
                raise BackendUnavailableError(f"engine library cannot be loaded: {exc}") from exc
            for name, (restype, argtypes) in EXPORTS.items():
                fn = getattr(handle, name)
                fn.restype = restype
                fn.argtypes = argtypes
            _lib = handle
    return _lib


def last_error() -> str:
    return lib().md200_last_error().decode(errors="replace")


def check(status: int) -> None:
    if status != 0:
        raise RuntimeError(last_error())


def default_options() -> Options:
    o = Options()
    lib().md200_default_options(ctypes.byref(o))
    return o


# cudaStreamLegacy: the legacy default stream.  The C ABI reads a NULL stream as
# "the engine's own stream", so handle 0 (torch's default stream) is passed as
# the legacy-stream handle instead.
CUDA_STREAM_LEGACY = 1


def _stream_arg(stream):
    if stream is None:
        return None
    return ctypes.c_void_p(int(stream) if int(stream) != 0 else CUDA_STREAM_LEGACY)


def ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


class Engine:
    """Owning handle of one md200_engine."""

    def __init__(self, device: int, capacity: int, layers: int, periods: int, nmodes: int,
                 options: Options):
        self.device, self.capacity, self.layers = int(device), int(capacity), int(layers)
        self.periods, self.nmodes = int(periods), int(nmodes)
        self.options = options
        handle = lib().md200_create(self.device, self.capacity, self.layers, self.periods, self.nmodes,
                                    ctypes.byref(options))
        if not handle:
            raise RuntimeError(last_error())
        self._handle = handle

    @property
    def handle(self):
        if not self._handle:
            raise RuntimeError("engine is closed")
        return self._handle

    def run(self, h, vp, vs, rho, periods, bounds, tol, accept, wave, group=False, prediction=False,
            continuity=False):
        """Host-array run; returns a dict of numpy outputs (``continuity_flags``
        [B, T] uint8 with `continuity`: the continuity screen's flags)."""
        B, L = h.shape
        T, nm = self.periods, self.nmodes
        arrays = [np.ascontiguousarray(x, dtype=np.float64) for x in (h, vp, vs, rho)]
        per = np.ascontiguousarray(periods, dtype=np.float64)
        bnd = None if bounds is None else np.ascontiguousarray(bounds, dtype=np.float64)
        out = dict(velocity=np.empty((B, nm, T)), flags=np.empty((B, T), np.uint32),
                   levels=np.empty((B, T), np.int32), counts=np.empty((B, T), np.int32),
                   bounds=np.empty((B, 2)), stats=np.zeros(STAT_COUNT, np.uint64))
        if group:
            out["group_velocity"] = np.empty((B, nm, T))
            out["group_velocity_flags"] = np.empty((B, nm, T), np.uint32)
        if prediction:
            out["prediction_flags"] = np.empty((B, T), np.uint32)
        if continuity:
            out["continuity_flags"] = np.empty((B, T), np.uint8)
        status = lib().md200_run(
            self.handle, *(ptr(a) for a in arrays), B, ptr(per), ptr(bnd), float(tol), float(accept),
            int(wave), ptr(out["velocity"]), ptr(out["flags"]), ptr(out["levels"]), ptr(out["counts"]),
            ptr(out.get("group_velocity")), ptr(out.get("group_velocity_flags")),
            ptr(out.get("prediction_flags")), ptr(out.get("continuity_flags")), ptr(out["bounds"]),
            ptr(out["stats"]), STAT_COUNT)
        check(status)
        out["stats"] = dict(zip(STAT_NAMES, (int(x) for x in out["stats"])))
        return out

    def run_device(self, h, vp, vs, rho, models, periods, bounds, tol, accept, wave, velocity, flags,
                   levels, counts, group=None, group_flags=None, prediction=None, bounds_out=None,
                   stats=None, stream=None, continuity=None):
        """Device-pointer run (integer addresses), enqueued on `stream` (a cudaStream_t
        address; None selects the engine's own stream, 0 the legacy default stream)."""
        c = ctypes.c_void_p
        status = lib().md200_run_device(
            self.handle, c(h), c(vp), c(vs), c(rho), int(models), c(periods), c(bounds) if bounds else None,
            float(tol), float(accept), int(wave), c(velocity), c(flags), c(levels), c(counts),
            c(group) if group else None, c(group_flags) if group_flags else None,
            c(prediction) if prediction else None, c(continuity) if continuity else None,
            c(bounds_out) if bounds_out else None, c(stats) if stats else None, _stream_arg(stream))
        check(status)

    def run_ragged(self, h, vp, vs, rho, period_offsets, periods, modes, tol, accept, wave, group=False,
                   bounds=None, continuity=False):
        """Ragged host-array run: model b has periods[period_offsets[b]:period_offsets[b+1]]
        and modes[b] modes.  Returns flat outputs: velocity (and group) as the
        concatenated [modes[b], T_b] blocks, trace arrays in CSR order."""
        arrays = [np.ascontiguousarray(x, dtype=np.float64) for x in (h, vp, vs, rho)]
        B = arrays[0].shape[0]
        off = np.ascontiguousarray(period_offsets, dtype=np.int32)
        per = np.ascontiguousarray(periods, dtype=np.float64)
        md = np.ascontiguousarray(modes, dtype=np.int32)
        if off.size != B + 1 or md.size != B:
            raise ValueError("period_offsets needs models + 1 entries and modes one per model")
        traces = int(off[-1])
        cells = int(np.sum(md.astype(np.int64) * np.diff(off)))
        out = dict(velocity=np.empty(cells), flags=np.empty(traces, np.uint32), levels=np.empty(traces, np.int32),
                   counts=np.empty(traces, np.int32), stats=np.zeros(STAT_COUNT, np.uint64))
        if group:
            out["group_velocity"] = np.empty(cells)
            out["group_velocity_flags"] = np.empty(cells, np.uint32)
        if continuity:
            out["continuity_flags"] = np.empty(traces, np.uint8)
        bnd = None if bounds is None else np.ascontiguousarray(bounds, dtype=np.float64)
        if bnd is not None and bnd.shape != (B, 2):
            raise ValueError("bounds must be [models, 2]")
        check(lib().md200_run_ragged(self.handle, *(ptr(a) for a in arrays), B, ptr(off), ptr(per), ptr(md),
                                     ptr(bnd), float(tol), float(accept), int(wave), ptr(out["velocity"]), ptr(out["flags"]),
                                     ptr(out["levels"]), ptr(out["counts"]), ptr(out.get("group_velocity")),
                                     ptr(out.get("group_velocity_flags")), ptr(out.get("continuity_flags")),
                                     ptr(out["stats"]), STAT_COUNT))
        out["stats"] = dict(zip(STAT_NAMES, (int(x) for x in out["stats"])))
        return out

    def run_ragged_device(self, h, vp, vs, rho, models, traces, period_offsets, periods, modes, out_offsets, tol,
                          accept, wave, velocity, flags, levels, counts, group=None, group_flags=None, stats=None,
                          stream=None, bounds=None, continuity=None):
        """Device-pointer ragged run (integer addresses), enqueued on `stream`."""
        c = ctypes.c_void_p
        opt = lambda x: c(x) if x else None
        check(lib().md200_run_ragged_device(self.handle, c(h), c(vp), c(vs), c(rho), int(models), int(traces),
                                            c(period_offsets), c(periods), c(modes), c(out_offsets), opt(bounds),
                                            float(tol),
                                            float(accept), int(wave), c(velocity), c(flags), c(levels), c(counts),
                                            opt(group), opt(group_flags), opt(continuity), opt(stats),
                                            _stream_arg(stream)))

    def jacobian(self, h, vp, vs, rho, periods, wave, velocity, group=None, want_group=True):
        """Host-array Jacobians of the roots `velocity` [B, nmodes, T]: returns
        (jac_phase, jac_group or None, failed) with jac_* [B, nmodes, T, 4, layers]
        (thickness, vp, vs, rho)."""
        arrays = [np.ascontiguousarray(x, dtype=np.float64) for x in (h, vp, vs, rho)]
        B, L = arrays[0].shape
        per = np.ascontiguousarray(periods, dtype=np.float64)
        vel = np.ascontiguousarray(velocity, dtype=np.float64)
        grp = None if group is None else np.ascontiguousarray(group, dtype=np.float64)
        shape = (B, self.nmodes, self.periods, 4, L)
        jc = np.empty(shape)
        ju = np.empty(shape) if want_group else None
        failed = ctypes.c_int()
        check(lib().md200_jacobian(self.handle, *(ptr(a) for a in arrays), B, ptr(per), int(wave), ptr(vel),
                                   ptr(grp), ptr(jc), ptr(ju), ctypes.byref(failed)))
        return jc, ju, int(failed.value)

    def vjp(self, h, vp, vs, rho, periods, wave, velocity, weight_phase=None, weight_group=None, group=None):
        """Host-array vector-Jacobian product: [4, B, layers] gradient."""
        arrays = [np.ascontiguousarray(x, dtype=np.float64) for x in (h, vp, vs, rho)]
        B, L = arrays[0].shape
        per = np.ascontiguousarray(periods, dtype=np.float64)
        vel = np.ascontiguousarray(velocity, dtype=np.float64)
        conv = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64)
        wc, wu, grp = conv(weight_phase), conv(weight_group), conv(group)
        grad = np.empty((4, B, L))
        check(lib().md200_vjp(self.handle, *(ptr(a) for a in arrays), B, ptr(per), int(wave), ptr(vel), ptr(grp),
                              ptr(wc), ptr(wu), ptr(grad)))
        return grad

    def jacobian_device(self, h, vp, vs, rho, models, periods, wave, velocity, jac_phase, group=None,
                        jac_group=None, stream=None):
        """Device-pointer Jacobians (integer addresses), enqueued on `stream`."""
        c = ctypes.c_void_p
        opt = lambda x: c(x) if x else None
        check(lib().md200_jacobian_device(self.handle, c(h), c(vp), c(vs), c(rho), int(models), c(periods),
                                          int(wave), c(velocity), opt(group), c(jac_phase), opt(jac_group),
                                          _stream_arg(stream)))

    def vjp_device(self, h, vp, vs, rho, models, periods, wave, velocity, grad, weight_phase=None,
                   weight_group=None, group=None, stream=None):
        """Device-pointer vector-Jacobian product into grad [4, models, layers]."""
        c = ctypes.c_void_p
        opt = lambda x: c(x) if x else None
        check(lib().md200_vjp_device(self.handle, c(h), c(vp), c(vs), c(rho), int(models), c(periods), int(wave),
                                     c(velocity), opt(group), opt(weight_phase), opt(weight_group), c(grad),
                                     _stream_arg(stream)))

    def graph_begin(self):
        """Start recording device-pointer runs (stream None) into a CUDA graph."""
        check(lib().md200_graph_begin(self.handle))

    def graph_end(self):
        """Finish the recording and instantiate the graph."""
        check(lib().md200_graph_end(self.handle))

    def graph_launch(self, stream=None):
        """Replay the recorded runs on `stream` (None = the engine's stream)."""
        check(lib().md200_graph_launch(self.handle, _stream_arg(stream)))

    def stage_times(self) -> dict:
        """Device milliseconds per stage of the last run (waits for it)."""
        ms = (ctypes.c_double * len(STAGES))()
        check(lib().md200_stage_times(self.handle, ms, len(STAGES)))
        return dict(zip(STAGES, list(ms)))

    def kernel_launches(self) -> int:
        return int(lib().md200_kernel_launches(self.handle))

    def close(self):
        if getattr(self, "_handle", None):
            lib().md200_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def device_count() -> int:
    return int(lib().md200_device_count())


def available(device: int = 0) -> bool:
    return bool(lib().md200_available(int(device)))


def set_device(device: int) -> None:
    check(lib().md200_set_device(int(device)))


def memory_info() -> tuple[int, int]:
    free, total = ctypes.c_size_t(), ctypes.c_size_t()
    check(lib().md200_memory_info(ctypes.byref(free), ctypes.byref(total)))
    return int(free.value), int(total.value)


def device_name(device: int = 0) -> str:
    buf = ctypes.create_string_buffer(256)
    check(lib().md200_device_name(int(device), buf, 256))
    return buf.value.decode()


def measure_peak(device: int = 0, fp64: bool = False) -> float:
    """Sustained FMA throughput of the device in flop/s (FP64 or FP32, non-tensor)."""
    out = ctypes.c_double()
    check(lib().md200_measure_peak(int(device), int(bool(fp64)), ctypes.byref(out)))
    return float(out.value)


def continuity_screen(periods, velocity, prediction=None, bilateral=True, device: int = 0):
    """The continuity screen on a result (md200_continuity_screen): (flags [B, T]
    uint8, suspect bool).  float32 velocities are screened as the reference screens
    float32 results (float32 comparisons and the 16-ULP rule)."""
    p = np.ascontiguousarray(periods, dtype=np.float64).ravel()
    v = np.asarray(velocity)
    single = v.dtype == np.float32
    v = np.ascontiguousarray(v, dtype=np.float64)
    if v.ndim != 3 or v.shape[2] != p.size:
        raise ValueError("continuity screening requires periods[T] and phases[B,K,T]")
    B, K, T = v.shape
    pred = None if prediction is None else np.ascontiguousarray(prediction, dtype=np.uint32)
    if pred is not None and pred.shape != (B, T):
        raise ValueError("prediction flags must have shape [B,T]")
    flags = np.empty((B, T), np.uint8)
    sus = ctypes.c_int()
    check(lib().md200_continuity_screen(int(device), ptr(p), T, ptr(v), B, K, ptr(pred), int(single),
                                        int(bool(bilateral)), ptr(flags), ctypes.byref(sus)))
    return flags, bool(sus.value)


def group_roots(h, vp, vs, rho, wave, period, roots, modes, close_rtol=.005):
    """Group velocities and flags of one model's ordered roots (arrays of length modes)."""
    arrays = [np.ascontiguousarray(x, dtype=np.float64).ravel() for x in (h, vp, vs, rho)]
    r = np.ascontiguousarray(roots, dtype=np.float64).ravel()
    group = np.empty(int(modes))
    flags = np.empty(int(modes), np.uint32)
    check(lib().md200_group_roots(*(ptr(a) for a in arrays), arrays[0].size, int(wave), float(period),
                                  ptr(r), r.size, int(modes), float(close_rtol), ptr(group), ptr(flags)))
    return group, flags


def reliability_plan(periods, max_log_period_gap: float):
    """The C plan builder (libm logarithms): (plan [T] PERIOD_PLAN, order [T] int32)."""
    p = np.ascontiguousarray(periods, dtype=np.float64).ravel()
    plan = np.zeros(p.size, PERIOD_PLAN)
    order = np.zeros(p.size, np.int32)
    check(lib().md200_reliability_plan(ptr(p), p.size, float(max_log_period_gap), ptr(plan), ptr(order)))
    return plan, order


def mode_reliability(velocity, plan, order, trace_flags=None, root_count=None, close_root_rtol=.005,
                     max_relative_step=.1, prediction_rtol=.05, device: int = 0):
    """Flags [B,K,T] uint16 and assessed [B,K,T] bool for host arrays (md200_mode_reliability)."""
    v = np.ascontiguousarray(velocity, dtype=np.float64)
    B, K, T = v.shape
    tf = None if trace_flags is None else np.ascontiguousarray(trace_flags, dtype=np.uint32)
    cnt = None if root_count is None else np.ascontiguousarray(root_count, dtype=np.int64)
    plan = np.ascontiguousarray(plan, dtype=PERIOD_PLAN)
    order = np.ascontiguousarray(order, dtype=np.int32)
    flags = np.empty(v.shape, np.uint16)
    assessed = np.empty(v.shape, np.uint8)
    check(lib().md200_mode_reliability(int(device), ptr(v), ptr(tf), ptr(cnt), B, K, T, ptr(plan), ptr(order),
                                       float(close_root_rtol), float(max_relative_step), float(prediction_rtol),
                                       ptr(flags), ptr(assessed)))
    return flags, assessed.astype(bool)


def mode_reliability_device(velocity, trace_flags, root_count, B, K, T, plan, order, close_root_rtol,
                            max_relative_step, prediction_rtol, flags, assessed, stream=None):
    """md200_mode_reliability_device on device pointers (ints); plan/order are host arrays."""
    plan = np.ascontiguousarray(plan, dtype=PERIOD_PLAN)
    order = np.ascontiguousarray(order, dtype=np.int32)
    check(lib().md200_mode_reliability_device(velocity, trace_flags, root_count, int(B), int(K), int(T), ptr(plan),
                                              ptr(order), float(close_root_rtol), float(max_relative_step),
                                              float(prediction_rtol), flags, assessed, _stream_arg(stream)))


def mode_reliability_planned(velocity, trace_flags, root_count, B, K, T, plan, order, close_root_rtol,
                             max_relative_step, prediction_rtol, flags, assessed, stream=None):
    """md200_mode_reliability_planned: every argument a device pointer (int)."""
    check(lib().md200_mode_reliability_planned(velocity, trace_flags, root_count, int(B), int(K), int(T), plan, order,
                                               float(close_root_rtol), float(max_relative_step),
                                               float(prediction_rtol), flags, assessed, _stream_arg(stream)))


def kernel_report(layers: int, single_precision: bool = False) -> dict:
    import json
    buf = ctypes.create_string_buffer(8192)
    check(lib().md200_kernel_report(int(layers), int(bool(single_precision)), buf, 8192))
    return json.loads(buf.value.decode())


class Uniform:
    """One md200_uniform object (the legacy uniform-grid path): a scan object
    after ``grid(nc)``, a refinement object after ``grid(nc, nmodes)``.  Plain
    handle methods over the C ABI; argument checks and the reference's error
    types live in the plugin's CoarseScan and Refine."""

    def __init__(self, models: int, layers: int):
        self.B, self.L = int(models), int(layers)
        self._h = lib().md200_uniform_create(self.B, self.L)
        if not self._h:
            raise RuntimeError(last_error())

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().md200_uniform_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def models(self, h, vp, vs, rho) -> None:
        a = [np.ascontiguousarray(x, dtype=np.float64) for x in (h, vp, vs, rho)]
        check(lib().md200_uniform_models(self._h, *(ptr(x) for x in a)))

    def periods(self, periods) -> None:
        p = np.ascontiguousarray(periods, dtype=np.float64)
        check(lib().md200_uniform_periods(self._h, int(p.size), ptr(p)))

    def grid(self, nc: int, nmodes: int = 0) -> None:
        check(lib().md200_uniform_grid(self._h, int(nc), int(nmodes)))

    def scan(self, cmin: float, cmax: float) -> None:
        check(lib().md200_uniform_scan(self._h, float(cmin), float(cmax)))

    def rows(self, nf: int, nc: int) -> np.ndarray:
        out = np.empty((self.B, nf, nc), np.float32)
        check(lib().md200_uniform_rows(self._h, ptr(out)))
        return out

    def set_rows(self, rows, cmin: float, cmax: float) -> None:
        r = np.ascontiguousarray(rows, dtype=np.float32)
        if r.size != self.B * np.prod(r.shape[1:]) or r.shape[0] != self.B:
            raise ValueError("rows must be [models, periods, nc]")
        check(lib().md200_uniform_set_rows(self._h, ptr(r), float(cmin), float(cmax)))

    def refine(self, scan: "Uniform", cmin, cmax, c_tol_rel, f_accept, nmodes) -> None:
        check(lib().md200_uniform_refine(self._h, scan._h, float(cmin), float(cmax), float(c_tol_rel),
                                         float(f_accept), int(nmodes)))

    @staticmethod
    def sync() -> None:
        check(lib().md200_uniform_sync())

    def velocity(self, nmodes: int, nf: int) -> np.ndarray:
        out = np.empty((self.B, nmodes, nf), np.float64)
        check(lib().md200_uniform_velocity(self._h, ptr(out)))
        return out

    def flags(self, nf: int) -> np.ndarray:
        out = np.empty((self.B, nf), np.uint32)
        check(lib().md200_uniform_flags(self._h, ptr(out)))
        return out

    def stats(self) -> dict:
        out = np.zeros(len(UNIFORM_STAT_NAMES), np.uint64)
        check(lib().md200_uniform_stats(self._h, ptr(out), out.size))
        return {k: int(v) for k, v in zip(UNIFORM_STAT_NAMES, out)}

    @staticmethod
    def iterations(dc: float, c_tol_rel: float, cmin: float) -> int:
        return int(lib().md200_uniform_iterations(float(dc), float(c_tol_rel), float(cmin)))

    @staticmethod
    def kernel_report(stage: int, layers: int, block: int = 256) -> str:
        buf = ctypes.create_string_buffer(512)
        check(lib().md200_uniform_kernel_report(int(stage), int(layers), int(block), buf, 512))
        return buf.value.decode()
