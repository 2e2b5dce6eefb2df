"""Command-line interface: ``python -m modisp_b200 {forward,check-modes,doctor}``.

The commands, options and NPZ keys of the reference's CLI (python/modisp/cli.py:9-113)
on this engine:

* ``forward INPUT --output OUT``: phase (and group) velocities from an NPZ holding
  ``thickness``, ``vp``, ``vs``, ``rho`` ([B, L] or [L]) and ``periods``.  A uniform
  input has ``periods`` [T] and writes the reference's output keys.  A ragged input
  adds ``period_offsets`` [B+1] (CSR: model b owns periods[offsets[b]:offsets[b+1]])
  and optionally ``nmodes`` [B]; it runs as one ragged batch
  (``modisp_b200.ragged.dispersion_ragged``) and writes flat CSR outputs: per trace
  ``trace_flags``, ``search_level``, ``root_count`` in period order, per model the
  ``[nmodes[b], T_b]`` block of ``phase_velocity`` (and ``group_velocity``) at
  ``out_offsets[b]``, with ``period_offsets``, ``periods`` and ``modes``.
* ``check-modes INPUT --output OUT``: cross-period mode-reliability checks of a
  uniform forward output (``modisp_b200.reliability``), the reference's output keys.
* ``doctor``: versions and device status as JSON.

Exit status as the reference's: 2 when any trace reports an unconverged search.
"""
from __future__ import annotations

import argparse
import json
import sys

import numpy as np

def _parser():
    from .api import DEFAULT_ACCURACY
    from . import __version__
    parser = argparse.ArgumentParser(prog="python -m modisp_b200")
    parser.add_argument("--version", action="version", version=__version__)
    sub = parser.add_subparsers(dest="command", required=True)
    sub.add_parser("doctor", help="show the engine library and device status")
    fw = sub.add_parser("forward", help="compute phase velocities from NPZ model/period arrays")
    fw.add_argument("input")
    fw.add_argument("--output", required=True)
    fw.add_argument("--wave", choices=["rayleigh", "love"], default="rayleigh")
    fw.add_argument("--backend", choices=["auto", "cuda", "b200"], default="auto")
    fw.add_argument("--precision", choices=["float64", "float32"], default="float64",
                    help="scan arithmetic (float32: FP32 scan, FP64 refinement)")
    fw.add_argument("--nmodes", type=int, default=3)
    fw.add_argument("--threads", type=int)
    fw.add_argument("--device", type=int, default=0)
    fw.add_argument("--cmin", type=float)
    fw.add_argument("--cmax", type=float)
    fw.add_argument("--accuracy", choices=["auto", "high", "balanced", "fast"], default=None,
                    help=f"search accuracy preset (default: {DEFAULT_ACCURACY})")
    fw.add_argument("--search-strategy", choices=["shape_adaptive", "qe_adaptive", "uniform"],
                    default="shape_adaptive")
    fw.add_argument("--sampling-rtol", type=float)
    fw.add_argument("--close-root-rtol", type=float, default=.005)
    fw.add_argument("--c-tol-rel", type=float)
    fw.add_argument("--secular", choices=["dunkin", "fast"], default=None)
    fw.add_argument("--refinement", choices=["legacy", "brent", "chandrupatla"], default=None)
    fw.add_argument("--love-strategy", choices=["phase", "scan"], default="phase")
    fw.add_argument("--group-velocity", action="store_true", help="compute FP64 group velocities")
    fw.add_argument("--group-rtol", type=float, default=.001)
    fw.add_argument("--frequency-strategy", choices=["independent", "anchor_continuation"], default="independent")
    fw.add_argument("--anchor-stride", type=int, default=4)
    fw.add_argument("--no-continuity-check", action="store_true",
                    help="disable the bilateral phase-curve recheck")
    fw.add_argument("--check-continuity", action="store_true",
                    help="save separate mode-reliability diagnostics (uniform inputs)")
    cm = sub.add_parser("check-modes", help="check an existing forward NPZ without solving again")
    cm.add_argument("input")
    cm.add_argument("--output", required=True)
    cm.add_argument("--max-relative-step", type=float, default=.1)
    cm.add_argument("--prediction-rtol", type=float, default=.05)
    cm.add_argument("--max-log-period-gap", type=float, default=.25)
    cm.add_argument("--close-root-rtol", type=float)
    return parser


def read_model(path):
    """(model arrays, periods, period_offsets or None, per-model nmodes or None) from an NPZ."""
    with np.load(path, allow_pickle=False) as src:
        model = {k: src[k] for k in ("thickness", "vp", "vs", "rho")}
        periods = src["periods"]
        offsets = src["period_offsets"] if "period_offsets" in src.files else None
        modes = src["nmodes"] if "nmodes" in src.files else None
    return model, periods, offsets, modes


def write_ragged(path, res, **extra):
    """Flat CSR outputs of a RaggedDispersion."""
    data = dict(period_offsets=res.period_offsets, periods=res.periods, modes=res.modes, out_offsets=res.out_offsets,
                phase_velocity=res.phase_velocity, trace_flags=res.trace_flags, search_level=res.search_level,
                root_count=res.root_count, wave=np.asarray(res.wave), layout=np.asarray("csr"))
    if res.group_velocity is not None:
        data.update(group_velocity=res.group_velocity, group_velocity_flags=res.group_velocity_flags)
    np.savez_compressed(path, **data, **extra)


# forward options that a ragged batch does not take, with their defaults
RAGGED_UNSUPPORTED = (("cmin", None), ("cmax", None), ("accuracy", None), ("sampling_rtol", None),
                      ("check_continuity", False), ("frequency_strategy", "independent"), ("threads", None))


def _forward_ragged(args, model, periods, offsets, modes):
    from .ragged import dispersion_ragged
    for name, default in RAGGED_UNSUPPORTED:
        if getattr(args, name) != default:
            raise ValueError(f"--{name.replace('_', '-')} is not available for ragged (period_offsets) inputs")
    nm = args.nmodes if modes is None else modes
    res = dispersion_ragged(model["thickness"], model["vp"], model["vs"], model["rho"], (offsets, periods), nmodes=nm,
                            wave=args.wave, precision="mixed" if args.precision == "float32" else "float64",
                            group_velocity=args.group_velocity,
                            c_tol_rel=args.c_tol_rel if args.c_tol_rel is not None else 1e-10, device=args.device)
    write_ragged(args.output, res, precision=np.asarray(args.precision))
    return 2 if np.any(res.trace_flags & 4) else 0


def _forward(args):
    from . import Solver
    from .reliability import check_mode_reliability
    model, periods, offsets, modes = read_model(args.input)
    if offsets is not None:
        return _forward_ragged(args, model, periods, offsets, modes)
    with Solver(backend=args.backend, threads=args.threads, device=args.device, cmin=args.cmin, cmax=args.cmax,
                accuracy=args.accuracy, close_root_rtol=args.close_root_rtol, c_tol_rel=args.c_tol_rel,
                search_strategy=args.search_strategy, sampling_rtol=args.sampling_rtol, secular=args.secular,
                refinement=args.refinement, love_strategy=args.love_strategy, precision=args.precision,
                group_velocity=args.group_velocity, group_rtol=args.group_rtol,
                frequency_strategy=args.frequency_strategy, anchor_stride=args.anchor_stride,
                continuity_check=not args.no_continuity_check) as solver:
        out = solver(**model, periods=periods, nmodes=args.nmodes, wave=args.wave)
        diagnostics = {}
        if args.check_continuity:
            check = check_mode_reliability(out, device=args.device)
            diagnostics.update(mode_reliability_flags=check.flags, continuity_assessed=check.assessed,
                               continuity_previous_index=check.previous_index,
                               continuity_sorted_order=check.sorted_order)
        if out.accuracy == "auto":
            diagnostics["auto_relaxed"] = out.auto_relaxed
            maximum = solver.stats().get("sampling_rtol_max")
            diagnostics["sampling_rtol_max"] = np.asarray(np.nan if maximum is None else maximum)
        if out.continuity_flags is not None:
            diagnostics["continuity_flags"] = out.continuity_flags
        if out.group_velocity is not None:
            diagnostics.update(group_velocity=out.group_velocity, group_velocity_flags=out.group_velocity_flags,
                               group_velocity_mask=out.group_velocity_mask,
                               group_velocity_valid=out.group_velocity_valid)
        if out.prediction_flags is not None:
            diagnostics["prediction_flags"] = out.prediction_flags
        np.savez_compressed(
            args.output, **diagnostics, refinement=np.asarray(out.refinement),
            love_strategy=np.asarray(out.love_strategy or ""), phase_velocity=out.phase_velocity, periods=out.period,
            mode_mask=out.mode_mask, status=out.status, trace_flags=out.trace_flags, search_bounds=out.search_bounds,
            search_level=out.search_level, root_count=out.root_count, backend=out.backend_used, wave=out.wave,
            precision=out.precision, accuracy=np.asarray(out.accuracy), numerical_flags=out.numerical_flags,
            approximate_search=out.approximate_search, close_root_mask=out.close_root_mask,
            potentially_ambiguous=out.potentially_ambiguous, mode_index_uncertain=out.mode_index_uncertain,
            close_root_risk=out.close_root_risk, close_root_rtol=np.asarray(out.close_root_rtol),
            search_strategy=np.asarray(out.search_strategy),
            sampling_rtol=np.asarray(np.nan if out.sampling_rtol is None else out.sampling_rtol),
            secular=np.asarray(out.secular), group_rtol=np.asarray(args.group_rtol),
            frequency_strategy=np.asarray(out.frequency_strategy),
            frequency_strategy_used=np.asarray(out.frequency_strategy_used),
            frequency_strategy_reason=np.asarray(out.frequency_strategy_reason),
            anchor_stride=np.asarray(out.anchor_stride))
    return 2 if np.any(out.trace_flags & 4) else 0


def _check_modes(args):
    from .reliability import check_mode_reliability
    with np.load(args.input, allow_pickle=False) as z:
        if "layout" in z.files and str(z["layout"]) == "csr":
            raise ValueError("check-modes takes a uniform forward output ([B, K, T] phase_velocity)")
        close = (args.close_root_rtol if args.close_root_rtol is not None
                 else float(z["close_root_rtol"]) if "close_root_rtol" in z.files else .005)
        check = check_mode_reliability(z["phase_velocity"], z["periods"], trace_flags=z["trace_flags"],
                                       root_count=z["root_count"], close_root_rtol=close,
                                       max_relative_step=args.max_relative_step, prediction_rtol=args.prediction_rtol,
                                       max_log_period_gap=args.max_log_period_gap)
    np.savez_compressed(args.output, continuity_flags=check.flags, continuity_assessed=check.assessed,
                        continuity_previous_index=check.previous_index, continuity_sorted_order=check.sorted_order)
    print(json.dumps(check.summary(), indent=2))
    return 0


def _doctor():
    from . import __version__, _native
    data = dict(version=__version__, python=sys.executable, library=str(_native.LIBRARY),
                abi_version=_native.ABI_VERSION, default_precision="float64", cuda_float32_available=True,
                accuracy_options=["auto", "high", "balanced", "fast"], default_continuity_check=True,
                default_group_velocity=False, default_group_rtol=.001)
    try:
        available = bool(_native.available(0))
        data.update(cuda_available=available, auto_backend="cuda" if available else "unavailable")
        if available:
            free, total = _native.memory_info()
            data.update(cuda_device=_native.device_name(0), free_device_bytes=free, total_device_bytes=total)
    except _native.BackendUnavailableError as exc:
        data.update(cuda_available=False, cuda_reason=str(exc), auto_backend="unavailable")
    print(json.dumps(data, indent=2))
    return 0


def main(argv=None):
    args = _parser().parse_args(argv)
    if args.command == "doctor":
        return _doctor()
    if args.command == "check-modes":
        return _check_modes(args)
    return _forward(args)


if __name__ == "__main__":
    raise SystemExit(main())
