"""``torch.autograd.Function`` over the per-frequency misfit Phi_f(s).

Forward: one oracle call (GPU assembly, factor, forward solve, source fit,
misfit).  Backward: the adjoint solve and the exact discrete slowness
gradient of wust_oracle.m:62-68, produced by the same C call and reused --
the factors are never recomputed for the backward.  ``curvature`` gives the
Gauss-Newton directional curvature of directional_curvature.m with the same
retained factors.
"""
from __future__ import annotations

import numpy as np
import torch

from .objective import Observations, directional_curvature, wust_oracle


class HelmholtzMisfit(torch.autograd.Function):
    @staticmethod
    def forward(ctx, slowness: torch.Tensor, obs: Observations, fi: int, cfg: dict):
        s = slowness.detach().to(torch.float64).cpu().numpy()
        c = 1.0 / s
        loss, grad, state = wust_oracle(c, obs, fi, cfg, nargout=3)
        ctx.state = state
        ctx.save_for_backward(torch.as_tensor(grad, dtype=slowness.dtype, device=slowness.device))
        return torch.tensor(loss, dtype=torch.float64, device=slowness.device)

    @staticmethod
    def backward(ctx, grad_out):
        (g,) = ctx.saved_tensors
        return (grad_out.to(g.dtype) * g), None, None, None


def misfit(slowness: torch.Tensor, obs: Observations, fi: int, cfg: dict) -> torch.Tensor:
    """Phi_f(s) with a hand-written backward (adjoint-state gradient)."""
    return HelmholtzMisfit.apply(slowness, obs, fi, cfg)


def misfit_and_state(slowness: torch.Tensor, obs: Observations, fi: int, cfg: dict):
    """(Phi_f, gradient, state) -- state feeds :func:`curvature`."""
    c = 1.0 / slowness.detach().to(torch.float64).cpu().numpy()
    return wust_oracle(c, obs, fi, cfg, nargout=3)


def curvature(state, direction) -> float:
    """d^T J^T J d with frozen source scales (directional_curvature.m)."""
    d = direction.detach().cpu().numpy() if isinstance(direction, torch.Tensor) else np.asarray(direction)
    return directional_curvature(state, d.astype(np.float64))
