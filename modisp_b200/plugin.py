"""The backend-plugin surface of modisp's CUDA extension, served by the B200 engine.

modisp selects a GPU backend by importing ``modisp_cuda`` and calling its
``load()``, which returns the extension module (python/modisp/_loader.py:15-28).
This module is that extension's interface, implemented over the engine's C ABI:
the same constants, module functions and ``QeSolver`` class with the same
argument meaning, return layout and error behaviour
(cpp/cuda/qe.cu:1124-1170, cpp/common/review_groups.hpp:39-63), and the legacy
uniform path's stage classes ``CoarseScan`` and ``Refine`` with ``STAT_NAMES``
(cpp/cuda/bindings.cpp:121-406) that modisp's ``search_strategy="uniform"``
drives (python/modisp/_legacy.py:300-340).  The package
``modisp_cuda`` at the repository root re-exports it, so an unmodified modisp
picks the engine with ``Solver(backend="cuda")``.

There is no CPU fallback: ``available()`` is False without an sm_100 GPU, and a
missing engine library raises BackendUnavailableError on load.
"""
from __future__ import annotations

import threading
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import _native

ABI_VERSION = 9
VERSION = "0.5.0"
SUPPORTS_FP32 = True
SUPPORTS_AUTO_ACCURACY = True
SUPPORTS_CANONICAL_LOWER = True
SUPPORTS_ROW_PERIODS = True
SUPPORTS_GROUP_VELOCITY = True
SUPPORTS_CONTINUATION = True
__file__ = str(_native.LIBRARY)


def available(device: int = 0) -> bool:
    """True when `device` is a usable sm_100 GPU (cpp/cuda/qe.cu:1131)."""
    try:
        return _native.available(device)
    except _native.BackendUnavailableError:
        return False


def set_device(device: int) -> None:
    _native.set_device(device)


def memory_info() -> tuple[int, int]:
    return _native.memory_info()


def device_name(device: int = 0) -> str:
    return _native.device_name(device)


def qe_kernel_report(L: int, accuracy: int = 0, shape: bool = False, single_precision: bool = False) -> dict:
    """Kernel attributes of the search engine (cpp/cuda/qe.cu:1143-1164)."""
    if not 1 <= int(L) <= 256:
        raise ValueError("L must be 1..256")
    report = _native.kernel_report(int(L), bool(single_precision))
    scan = report["kernels"]["scan_fp32" if single_precision else "scan_fp64"]
    return dict(registers_per_thread=scan["registers"], static_shared_bytes=scan["static_shared_bytes"],
                local_bytes_per_thread=scan["local_bytes"], search_block_threads=128,
                max_active_blocks_per_sm=scan["blocks_per_sm_at_128"],
                dynamic_shared_bytes=scan["dynamic_shared_bytes"],
                search_kernel="b200_scan_fp32" if single_precision else "b200_scan_fp64",
                kernels=report["kernels"])


def love_phase_kernel_report(L: int, single_precision: bool = False) -> dict:
    """Love traces use the same scan kernel as Rayleigh traces."""
    return qe_kernel_report(L, 0, True, single_precision)


def _review_groups(packed, layers, modes, wave, secular, period, lo, hi, rtol, close_rtol):
    """Group velocities of a repaired trace: (velocities [modes], flags [modes], evaluations)."""
    packed = np.ascontiguousarray(packed, dtype=np.float64)
    layers, modes = int(layers), int(modes)
    if packed.ndim != 1 or not 1 <= layers <= 256 or not 1 <= modes <= 256 or \
            packed.size < 4 * layers or packed.size > 4 * layers + 256 or not period > 0:
        raise ValueError("invalid review trace")
    h, vp, vs, rho = (packed[i * layers:(i + 1) * layers] for i in range(4))
    roots = packed[4 * layers:]
    group, flags = _native.group_roots(h, vp, vs, rho, int(wave), float(period), roots, modes,
                                       float(close_rtol))
    return group, flags, int(np.count_nonzero(flags == 0))


_cast_pool = None
_cast_lock = threading.Lock()


def _pool():
    global _cast_pool
    with _cast_lock:
        if _cast_pool is None:
            _cast_pool = ThreadPoolExecutor(8, thread_name_prefix="md200-cast")
    return _cast_pool


def _count_nonzero(a):
    """np.count_nonzero of a large array, counted in slices on 8 threads (numpy
    releases the GIL while counting)."""
    if a.size < 1 << 20:
        return int(np.count_nonzero(a))
    flat = a.reshape(-1)
    step = -(-flat.size // 8)
    return int(sum(_pool().map(lambda i: np.count_nonzero(flat[i * step:(i + 1) * step]), range(8))))


def _to_float32(a):
    """float32 copy of a float64 array (the reference's FP32-mode output type),
    converted in slices on 8 threads for large arrays: numpy releases the GIL
    while casting, and the rounding is the same as astype's."""
    if a.size < 1 << 20:
        return a.astype(np.float32)
    out = np.empty(a.shape, np.float32)
    src, dst = a.reshape(-1), out.reshape(-1)
    step = -(-src.size // 8)
    list(_pool().map(lambda i: np.copyto(dst[i * step:(i + 1) * step], src[i * step:(i + 1) * step],
                                         casting="same_kind"), range(8)))
    return out


class QeSolver:
    """Engine with a fixed capacity and geometry (cpp/cuda/qe.cu:978-1036).

    Arguments follow the reference constructor: B (capacity), L, nf, nmodes,
    accuracy {0 high, 1 balanced, 2 fast, 3 uniform, 4 auto}, period_threshold,
    close_root_rtol, shape, sampling_rtol, secular {0, 1}, refinement {0, 1, 2},
    love_phase, single_precision, group_velocity, group_rtol, continuation,
    anchor_stride.  Engine keywords (scan_density, log_points, warps_per_block,
    blocks_per_sm, continuity_check, device) may follow.
    """

    def __init__(self, B, L, nf, nmodes, accuracy=0, period_threshold=0., close_root_rtol=.005,
                 shape=False, sampling_rtol=.001, secular=0, refinement=1, love_phase=1,
                 single_precision=False, group_velocity=False, group_rtol=.001, continuation=False,
                 anchor_stride=4, *, scan_density=0., log_points=0, warps_per_block=0, blocks_per_sm=0,
                 continuity_check=True, device=None):
        if int(B) < 1 or not 1 <= int(L) <= 256 or int(nf) < 1 or not 1 <= int(nmodes) <= 256:
            raise ValueError("invalid QE geometry")
        if int(refinement) not in (0, 1, 2) or int(secular) not in (0, 1):
            raise ValueError("invalid refinement or secular selector")
        if continuation and int(anchor_stride) < 2:
            raise ValueError("anchor_stride must be at least 2")
        o = _native.default_options()
        o.accuracy = int(accuracy)
        o.period_threshold = float(period_threshold)
        o.close_root_rtol = float(close_root_rtol)
        o.shape = int(bool(shape))
        o.sampling_rtol = float(sampling_rtol)
        o.secular = int(secular)
        o.refinement = int(refinement)
        o.love_phase = int(love_phase)
        o.single_precision = int(bool(single_precision))
        o.group_velocity = int(bool(group_velocity))
        o.group_rtol = float(group_rtol)
        o.continuation = int(bool(continuation))
        o.anchor_stride = int(anchor_stride)
        o.scan_density = float(scan_density)
        o.log_points = int(log_points)
        o.warps_per_block = int(warps_per_block)
        o.blocks_per_sm = int(blocks_per_sm)
        o.continuity_check = int(bool(continuity_check))
        if device is None:
            device = _current_device
        self.capacity, self.layers, self.nf, self.nmodes = int(B), int(L), int(nf), int(nmodes)
        self.single_precision = bool(single_precision)
        self.group_velocity = bool(group_velocity)
        self.continuation = bool(continuation)
        self._engine = _native.Engine(int(device), self.capacity, self.layers, self.nf, self.nmodes, o)

    def run(self, thickness, vp, vs, rho, periods, bounds, c_tol_rel=1e-6, f_accept=1.0, wave=0,
            automatic=False, profile=False, canonical_lower=False):
        """Solve one chunk (cpp/cuda/qe.cu:1060-1119).

        Returns (velocity [B', nmodes, nf], flags [B', nf] uint32, stats dict,
        levels [B', nf] int32, counts [B', nf] int32, extras) with extras holding
        group_velocity / group_velocity_flags (or None) and prediction_flags (or None).
        """
        del automatic, canonical_lower  # the engine's window is the one passed in
        h = np.ascontiguousarray(thickness, dtype=np.float64)
        if h.ndim != 2 or h.shape[1] != self.layers or not 1 <= h.shape[0] <= self.capacity:
            raise ValueError("model shapes differ from the engine geometry")
        arrays = [np.ascontiguousarray(x, dtype=np.float64) for x in (vp, vs, rho)]
        if any(a.shape != h.shape for a in arrays):
            raise ValueError("model shapes differ")
        per = np.ascontiguousarray(periods, dtype=np.float64)
        bnd = np.ascontiguousarray(bounds, dtype=np.float64)
        if bnd.shape != (h.shape[0], 2):
            raise ValueError("bounds must be [B, 2]")
        B = h.shape[0]
        if per.ndim == 2 and per.shape == (B, 1) and self.nf == 1:
            # one period per model (cpp/cuda/qe.cu:1069-1070): a ragged batch of one trace per model
            out = self._engine.run_ragged(h, *arrays, np.arange(B + 1, dtype=np.int32), per[:, 0],
                                          np.full(B, self.nmodes, np.int32), c_tol_rel, f_accept, int(wave),
                                          group=self.group_velocity, bounds=bnd)
            shape = (B, self.nmodes, 1)
            out["velocity"] = out["velocity"].reshape(shape)
            if self.group_velocity:
                out["group_velocity"] = out["group_velocity"].reshape(shape)
                out["group_velocity_flags"] = out["group_velocity_flags"].reshape(shape)
            for k in ("flags", "levels", "counts"):
                out[k] = out[k].reshape(B, 1)
        else:
            if per.ndim != 1 or per.size != self.nf:
                raise ValueError("periods must be a 1-D array of the engine's period count")
            out = self._engine.run(h, *arrays, per, bnd, c_tol_rel, f_accept, int(wave),
                                   group=self.group_velocity, prediction=self.continuation)
        velocity = _to_float32(out["velocity"]) if self.single_precision else out["velocity"]
        stats = dict(out["stats"])
        stats.update(strategy="b200_scan", capacity=self.capacity)
        if self.group_velocity:
            # the counters the reference's continuity review adds to
            # (python/modisp/_continuity.py:112-119, :136-137; cpp/cpu/solver.cpp:748-749)
            stats["group_evaluations"] = int(stats.get("group_roots", 0))
            stats["group_invalid"] = _count_nonzero(out["group_velocity_flags"])
        extras = dict(group_velocity=out.get("group_velocity"),
                      group_velocity_flags=out.get("group_velocity_flags"),
                      prediction_flags=out.get("prediction_flags"))
        return velocity, out["flags"], stats, out["levels"], out["counts"], extras

    def close(self):
        if getattr(self, "_engine", None) is not None:
            self._engine.close()
            self._engine = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# Counter names of the legacy uniform path's Refine.stats(), in order
# (cpp/cuda/bindings.cpp:58-59, exported as the module's STAT_NAMES at :348-351).
STAT_NAMES = _native.UNIFORM_STAT_NAMES


def _as_2d(obj, rows, cols, name):
    """Contiguous float64 [rows, cols] (cpp/cuda/bindings.cpp:79-93: TypeError when
    not array-like, ValueError on a shape mismatch)."""
    try:
        a = np.ascontiguousarray(obj, dtype=np.float64)
    except (TypeError, ValueError) as exc:
        raise TypeError(f"{name} must be an array-like of real numbers") from exc
    if a.ndim != 2 or a.shape != (rows, cols):
        raise ValueError(f"{name} must have shape ({rows}, {cols}), got {a.shape}")
    return a


def _as_periods(periods):
    try:
        p = np.ascontiguousarray(periods, dtype=np.float64)
    except (TypeError, ValueError):
        p = None
    if p is None or p.ndim != 1 or p.size == 0:
        raise ValueError("periods must be a non-empty 1-D array")
    return p


class _UniformStage:
    """State shared by the legacy path's two stage objects: B models of L rows,
    the uploaded periods and the allocated grid."""

    def __init__(self, B, L):
        self._u = _native.Uniform(int(B), int(L))
        self.B, self.L = int(B), int(L)
        self.nf = self.nc = 0
        self._uploaded = False

    def upload_models(self, thickness, vp, vs, rho):
        arrays = [_as_2d(x, self.B, self.L, n) for x, n in ((thickness, "thickness"), (vp, "vp"), (vs, "vs"),
                                                           (rho, "rho"))]
        self._u.models(*arrays)
        self._uploaded = True

    def upload_periods(self, periods):
        p = _as_periods(periods)
        self._u.periods(p)
        if p.size != self.nf:
            self.nc = 0  # outputs sized for another period count are dropped
            if hasattr(self, "nmodes"):
                self.nmodes = 0
        self.nf = int(p.size)

    def sync(self):
        _native.Uniform.sync()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return None

    def close(self):
        self._u.close()


class CoarseScan(_UniformStage):
    """Stage 1 of the legacy uniform path: FP32 secular values over a (period,
    velocity) grid (cpp/cuda/bindings.cpp:121-196, cpp/cuda/coarse_scan.cu)."""

    def __init__(self, B, L):
        super().__init__(B, L)
        self._range = None

    def allocate(self, nc):
        self._u.grid(int(nc), 0)
        self.nc = int(nc)

    def run(self, cmin, cmax, block=256, sync=False):
        del block  # the kernel's block shape is fixed; results do not depend on it
        if not self._uploaded:
            raise RuntimeError("upload_models() first")
        self._u.scan(cmin, cmax)
        self._range = (float(cmin), float(cmax))
        if sync:
            self.sync()

    def download(self):
        if not self.nc:
            raise RuntimeError("allocate() first")
        return self._u.rows(self.nf, self.nc)

    def scan(self, cmin, cmax, block=256):
        self.run(cmin, cmax, block, True)
        return self.download()

    def kernel_report(self, block=256):
        return _native.Uniform.kernel_report(0, self.L, block)


class Refine(_UniformStage):
    """Stages 2-3 of the legacy uniform path: roots located from a CoarseScan's
    values and bisected in FP64 (cpp/cuda/bindings.cpp:200-345, cpp/cuda/refine.cu)."""

    def __init__(self, B, L):
        super().__init__(B, L)
        self.nmodes = 0

    def allocate(self, nc, nmodes):
        self._u.grid(int(nc), int(nmodes))
        self.nc, self.nmodes = int(nc), int(nmodes)

    def run(self, scan, cmin, cmax, c_tol_rel=1e-6, f_accept=1.0, nmodes=0, block=256, sync=True):
        del block
        if not self.nf:
            raise RuntimeError("upload_periods() first")
        if not self.nmodes:
            raise RuntimeError("allocate() first")
        if (scan.B, scan.L, scan.nf, scan.nc) != (self.B, self.L, self.nf, self.nc):
            raise ValueError(f"scan and refine geometries differ: scan has B={scan.B} L={scan.L} nf={scan.nf} "
                             f"nc={scan.nc}, refine has B={self.B} L={self.L} nf={self.nf} nc={self.nc}")
        if scan._range is None:
            raise ValueError("this scan has not been run, so its rows hold nothing to refine; call run() on it "
                             "first")
        if scan._range != (float(cmin), float(cmax)):
            raise ValueError(f"scan and refine ranges differ: the scan ran over {scan._range}, the refinement was "
                             f"given ({float(cmin)}, {float(cmax)}); the range sets the grid spacing, so every "
                             "grid point would move")
        self._u.refine(scan._u, cmin, cmax, c_tol_rel, f_accept, nmodes)
        if int(nmodes) > 0:
            self.nmodes = int(nmodes)
        if sync:
            self.sync()

    def download(self):
        if not self.nmodes:
            raise RuntimeError("allocate() first")
        return self._u.velocity(self.nmodes, self.nf)

    def stats(self):
        return self._u.stats()

    def flags(self):
        if not self.nf or not self.nmodes:
            raise RuntimeError("allocate() first")
        return self._u.flags(self.nf)

    def kernel_report(self, block=256):
        return _native.Uniform.kernel_report(1, self.L, block)


_current_device = 0


def _track_device(device: int) -> None:
    global _current_device
    _current_device = int(device)


_set_device = set_device


def set_device(device: int) -> None:  # noqa: F811 - records the device for new engines
    _set_device(device)
    _track_device(device)
