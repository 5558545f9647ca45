"""``torch.autograd.Function`` over the per-frequency misfit Phi_f(s).

Forward: one oracle call (GPU assembly, factor, forward solve, source fit,
misfit) on the slowness as a CUDA tensor -- nothing crosses to the host but
the scalar misfit.  When the slowness needs a gradient the same call also
runs the adjoint solve and the exact discrete slowness gradient of
wust_oracle.m:62-68 and keeps its state; without one it runs the forward
solve only (wust_oracle.m:5-6: the number of outputs selects the work).
Backward: returns that gradient -- the factors are never recomputed.  The
gradient is itself differentiable: its derivative along a vector v is the
Gauss-Newton Hessian-vector product Re(J^H J v) with the source scales frozen
(the product whose quadratic form is directional_curvature.m's curvature),
one more forward and one more adjoint solve on the retained factors, so
``torch.autograd.grad`` of the gradient gives curvature-vector products.
"""
from __future__ import annotations

import numpy as np
import torch

from .objective import Observations, directional_curvature, gauss_newton_product, wust_oracle


class _MisfitGradient(torch.autograd.Function):
    """g(s) as a node of the graph; its backward is the Gauss-Newton product."""

    @staticmethod
    def forward(ctx, slowness: torch.Tensor, grad: torch.Tensor, state):
        ctx.state = state
        return grad.to(slowness.dtype).clone()

    @staticmethod
    def backward(ctx, v):
        hv, _ = gauss_newton_product(ctx.state, v.to(torch.float64))
        return hv.to(v.dtype), None, None


class HelmholtzMisfit(torch.autograd.Function):
    @staticmethod
    def forward(ctx, slowness: torch.Tensor, obs: Observations, fi: int, cfg: dict):
        if not slowness.is_cuda:
            raise ValueError("the slowness must be a CUDA tensor")
        c = 1.0 / slowness.detach().to(torch.float64)
        if ctx.needs_input_grad[0]:
            loss, grad, state = wust_oracle(c, obs, fi, cfg, nargout=3)
            ctx.state = state
            ctx.grad = grad
            ctx.save_for_backward(slowness)
        else:
            loss = wust_oracle(c, obs, fi, cfg, nargout=1)
        return torch.tensor(loss, dtype=torch.float64, device=slowness.device)

    @staticmethod
    def backward(ctx, grad_out):
        (slowness,) = ctx.saved_tensors
        g = _MisfitGradient.apply(slowness, ctx.grad, ctx.state)
        return grad_out.to(g.dtype) * g, None, None, None


def misfit(slowness: torch.Tensor, obs: Observations, fi: int, cfg: dict) -> torch.Tensor:
    """Phi_f(s) with a hand-written backward (adjoint-state gradient), twice
    differentiable in the Gauss-Newton sense."""
    return HelmholtzMisfit.apply(slowness, obs, fi, cfg)


def misfit_and_state(slowness: torch.Tensor, obs: Observations, fi: int, cfg: dict):
    """(Phi_f, gradient, state) -- state feeds :func:`curvature`; the slowness
    stays on the device when it is a CUDA tensor."""
    s = slowness.detach().to(torch.float64)
    c = 1.0 / s if s.is_cuda else 1.0 / s.numpy()
    return wust_oracle(c, obs, fi, cfg, nargout=3)


def curvature(state, direction) -> float:
    """d^T J^T J d with frozen source scales (directional_curvature.m)."""
    d = direction.detach().cpu().numpy() if isinstance(direction, torch.Tensor) else np.asarray(direction)
    return directional_curvature(state, d.astype(np.float64))
