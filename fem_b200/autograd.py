"""torch.autograd wrapper of the engine (a thin gradcheck binding).

``homogenize(rho, engine)`` returns C^H as a differentiable function of the
density field: the forward pass is femh_homogenize, the backward pass is the
hand-written adjoint kernel (femh_homogenize_grad) applied to the incoming
dL/dC -- the operator is self-adjoint, so no second solve runs.  This mirrors
the reference's FEM3DFun::setParam / df pair (fast_fem/FEM3DFun.cpp:128-268),
where df is the analytic gradient of a loss on G = C^H.
"""
from __future__ import annotations

import numpy as np
import torch

from .femh import Engine


def _solve(engine: Engine, rho_c: torch.Tensor) -> np.ndarray:
    C, _ = engine.homogenize(rho_c if rho_c.is_cuda else rho_c.numpy())
    engine._autograd_rho = rho_c.clone()
    return C


class HomogenizeFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, rho: torch.Tensor, engine: Engine):
        if rho.dtype != torch.float64:
            raise TypeError("rho must be float64")
        rho_c = rho.detach().contiguous()
        C = _solve(engine, rho_c)
        ctx.save_for_backward(rho_c)
        ctx.engine = engine
        ctx.rho_device = rho.device
        ctx.shape = tuple(rho.shape)
        return torch.from_numpy(np.ascontiguousarray(C)).to(rho.device)

    @staticmethod
    def backward(ctx, grad_C: torch.Tensor):
        dLdC = grad_C.detach().cpu().numpy().astype(np.float64)
        (rho_c,) = ctx.saved_tensors
        last = getattr(ctx.engine, "_autograd_rho", None)
        if last is None or last.shape != rho_c.shape or not torch.equal(last, rho_c):
            _solve(ctx.engine, rho_c)   # another cell was solved since: restore this one's fields
        g = ctx.engine.grad(dLdC)   # adjoint kernel on the resident solved fields
        return torch.from_numpy(g.reshape(ctx.shape)).to(ctx.rho_device), None


def homogenize(rho: torch.Tensor, engine: Engine) -> torch.Tensor:
    """C^H (6x6, float64 tensor) of the periodic cell rho with autograd support.

    The backward pass reuses the engine's resident solved fields when the
    engine's last solve was this rho, and re-solves otherwise."""
    return HomogenizeFn.apply(rho, engine)
