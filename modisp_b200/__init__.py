"""modisp_b200: a B200-native (sm_100a) engine for multimode Rayleigh/Love dispersion.

Drop-in for modisp's GPU backend: the public API of modisp (``dispersion``,
``dispersion_batch``, ``Solver``, ``DispersionBatch`` and its flags) runs on
hand-written CUDA kernels behind a C ABI (``include/modisp_b200.h``), and the
package ``modisp_cuda`` serves the same engine to an unmodified modisp through
its backend-plugin contract.
"""
from .api import (  # noqa: F401
    DEFAULT_ACCURACY, DispersionBatch, GroupVelocityFlag, PredictionFlag, SolveStatus, Solver,
    dispersion, dispersion_batch, release, device_name,
    TRACE_UNRESOLVED_BRACKET, TRACE_RELOCATED, TRACE_SEARCH_UNCONVERGED, TRACE_WORKSPACE_LIMIT,
    TRACE_NEAR_CUTOFF, TRACE_NONFINITE, TRACE_REFINEMENT_FAILED, TRACE_F_REJECTED, TRACE_RANGE_TRUNCATED,
    TRACE_SAMPLING_UNCERTAIN, TRACE_ROOT_CONFLICT, TRACE_APPROXIMATE_SEARCH, TRACE_CLOSE_ROOT_RISK,
    TRACE_ADAPTIVE_FALLBACK, TRACE_LOVE_PHASE_FALLBACK, TRACE_FP64_REPAIR, TRACE_CONTINUATION_APPROXIMATE,
    TRACE_AUTO_RELAXED, LEVEL_FP64_SCAN, LEVEL_FP32_SCAN, LEVEL_FP32_REPAIRED, LEVEL_CONTINUATION,
)
from ._native import BackendUnavailableError  # noqa: F401
from .reliability import ModeReliability, ModeReliabilityFlag, check_mode_reliability  # noqa: F401

__version__ = "0.5.0"
