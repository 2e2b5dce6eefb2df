"""Differentiable phase and group velocities: a torch.autograd.Function over the engine.

    solver = DifferentiableSolver(capacity=B, layers=L, periods=periods, nmodes=3)
    phase, group = solver(thickness, vp, vs, rho)          # CUDA float64 [B, L] tensors
    loss = ((phase - observed)[mask] ** 2).sum()
    loss.backward()                                        # thickness.grad, vp.grad, ...

Forward: one engine run (root search, refinement, group velocity) on the
tensors' device memory, on the current torch stream.  Backward: the engine's
adjoint sweep (``md200_vjp_device``) turns the cotangents of every phase and
group velocity into the gradient with respect to each row's thickness, Vp, Vs
and density -- the implicit-function derivatives dc/dm = -F_m / F_c and their
group-velocity counterparts -- without forming the Jacobians; the layer
recurrences are recomputed in the backward pass, nothing but the inputs and
the roots is saved.  ``jacobian`` returns the full Jacobians instead.

PyTorch is the plumbing here (device memory, streams, autograd); every
derivative is computed by the engine's CUDA kernels.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _native

WAVES = {"rayleigh": 0, "love": 1}


def _stream(device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def _check(x: torch.Tensor, name: str, shape=None) -> torch.Tensor:
    if not isinstance(x, torch.Tensor) or not x.is_cuda:
        raise TypeError(f"{name} must be a CUDA tensor")
    if x.dtype != torch.float64:
        raise TypeError(f"{name} must be float64")
    if shape is not None and tuple(x.shape) != tuple(shape):
        raise ValueError(f"{name} has shape {tuple(x.shape)}, expected {tuple(shape)}")
    return x.contiguous()


class DifferentiableSolver:
    """One engine (fixed layers, periods and modes) whose outputs carry gradients.

    ``precision``: "float64" (FP64 scan) or "mixed" (FP32 scan, FP64 refinement);
    roots, group velocities and derivatives are FP64 either way.
    """

    def __init__(self, capacity: int, layers: int, periods, nmodes: int, wave: str = "rayleigh",
                 precision: str = "mixed", c_tol_rel: float = 1e-10, device: int | None = None):
        if wave not in WAVES:
            raise ValueError("wave must be 'rayleigh' or 'love'")
        if precision not in ("float64", "mixed"):
            raise ValueError("precision must be 'float64' or 'mixed'")
        self.device = torch.cuda.current_device() if device is None else int(device)
        per = np.ascontiguousarray(periods, dtype=np.float64).ravel()
        self.periods = torch.tensor(per, dtype=torch.float64, device=f"cuda:{self.device}")
        self.capacity, self.layers, self.nmodes = int(capacity), int(layers), int(nmodes)
        self.wave = WAVES[wave]
        self.tol = float(c_tol_rel)
        o = _native.default_options()
        o.single_precision = 1 if precision == "mixed" else 0
        o.group_velocity = 1
        self.engine = _native.Engine(self.device, self.capacity, self.layers, per.size, self.nmodes, o)

    def _inputs(self, thickness, vp, vs, rho):
        B = thickness.shape[0] if thickness.dim() == 2 else -1
        shape = (B, self.layers)
        if B < 1 or B > self.capacity:
            raise ValueError(f"model count {B} outside 1..{self.capacity}")
        return [_check(x, n, shape) for x, n in ((thickness, "thickness"), (vp, "vp"), (vs, "vs"), (rho, "rho"))]

    def solve(self, thickness, vp, vs, rho):
        """Roots and group velocities (no autograd): dict of CUDA tensors."""
        h, a, b, r = self._inputs(thickness, vp, vs, rho)
        B, T, nm = h.shape[0], self.periods.numel(), self.nmodes
        dev = h.device
        out = dict(velocity=torch.empty((B, nm, T), dtype=torch.float64, device=dev),
                   group_velocity=torch.empty((B, nm, T), dtype=torch.float64, device=dev),
                   group_velocity_flags=torch.empty((B, nm, T), dtype=torch.int32, device=dev),
                   flags=torch.empty((B, T), dtype=torch.int32, device=dev),
                   levels=torch.empty((B, T), dtype=torch.int32, device=dev),
                   counts=torch.empty((B, T), dtype=torch.int32, device=dev))
        self.engine.run_device(h.data_ptr(), a.data_ptr(), b.data_ptr(), r.data_ptr(), B, self.periods.data_ptr(),
                               None, self.tol, 1., self.wave, out["velocity"].data_ptr(), out["flags"].data_ptr(),
                               out["levels"].data_ptr(), out["counts"].data_ptr(), out["group_velocity"].data_ptr(),
                               out["group_velocity_flags"].data_ptr(), stream=_stream(dev))
        return out

    def __call__(self, thickness, vp, vs, rho):
        """(phase [B, nmodes, T], group [B, nmodes, T]); NaN where no root."""
        return _Dispersion.apply(thickness, vp, vs, rho, self)

    def jacobian(self, thickness, vp, vs, rho, velocity=None, group=None):
        """Full Jacobians of the roots: (dc/dm, dU/dm), each [B, nmodes, T, 4, L]
        (m = thickness, vp, vs, rho).  Solves first unless the roots are given."""
        h, a, b, r = self._inputs(thickness, vp, vs, rho)
        if velocity is None:
            res = self.solve(h, a, b, r)
            velocity, group = res["velocity"], res["group_velocity"]
        B, T = h.shape[0], self.periods.numel()
        vel = _check(velocity, "velocity", (B, self.nmodes, T))
        grp = None if group is None else _check(group, "group", (B, self.nmodes, T))
        shape = (B, self.nmodes, T, 4, self.layers)
        jc = torch.empty(shape, dtype=torch.float64, device=h.device)
        ju = torch.empty(shape, dtype=torch.float64, device=h.device)
        self.engine.jacobian_device(h.data_ptr(), a.data_ptr(), b.data_ptr(), r.data_ptr(), B,
                                    self.periods.data_ptr(), self.wave, vel.data_ptr(), jc.data_ptr(),
                                    group=grp.data_ptr() if grp is not None else None, jac_group=ju.data_ptr(),
                                    stream=_stream(h.device))
        return jc, ju

    def vjp(self, thickness, vp, vs, rho, velocity, group, weight_phase=None, weight_group=None):
        """sum over cells of weight_phase dc/dm + weight_group dU/dm: [4, B, L]."""
        h, a, b, r = self._inputs(thickness, vp, vs, rho)
        B, T = h.shape[0], self.periods.numel()
        cells = (B, self.nmodes, T)
        vel = _check(velocity, "velocity", cells)
        grp = None if group is None else _check(group, "group", cells)
        wc = None if weight_phase is None else _check(weight_phase, "weight_phase", cells)
        wu = None if weight_group is None else _check(weight_group, "weight_group", cells)
        grad = torch.empty((4, B, self.layers), dtype=torch.float64, device=h.device)
        if wc is None and wu is None:
            return grad.zero_()
        self.engine.vjp_device(h.data_ptr(), a.data_ptr(), b.data_ptr(), r.data_ptr(), B, self.periods.data_ptr(),
                               self.wave, vel.data_ptr(), grad.data_ptr(),
                               weight_phase=wc.data_ptr() if wc is not None else None,
                               weight_group=wu.data_ptr() if wu is not None else None,
                               group=grp.data_ptr() if grp is not None else None, stream=_stream(h.device))
        return grad

    def close(self):
        self.engine.close()


class _Dispersion(torch.autograd.Function):
    @staticmethod
    def forward(ctx, thickness, vp, vs, rho, solver):
        res = solver.solve(thickness, vp, vs, rho)
        vel, grp = res["velocity"], res["group_velocity"]
        ctx.solver = solver
        ctx.save_for_backward(thickness, vp, vs, rho, vel, grp)
        return vel, grp

    @staticmethod
    def backward(ctx, grad_phase, grad_group):
        thickness, vp, vs, rho, vel, grp = ctx.saved_tensors
        g = ctx.solver.vjp(thickness, vp, vs, rho, vel, grp,
                           None if grad_phase is None else grad_phase.contiguous(),
                           None if grad_group is None else grad_group.contiguous())
        return g[0], g[1], g[2], g[3], None


def misfit(phase, group, phase_obs, group_obs, group_weight: float = 1.0):
    """L2 misfit over the cells where both the prediction and the observation
    exist: sum (c - c_obs)^2 + group_weight * sum (U - U_obs)^2."""
    mc = torch.isfinite(phase) & torch.isfinite(phase_obs)
    mu = torch.isfinite(group) & torch.isfinite(group_obs) & mc
    return ((phase - phase_obs)[mc] ** 2).sum() + group_weight * ((group - group_obs)[mu] ** 2).sum()
