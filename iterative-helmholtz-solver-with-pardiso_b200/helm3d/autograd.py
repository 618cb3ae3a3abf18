"""torch.autograd binding of the misfit gradient (for tests and for callers
that drive an inversion from PyTorch).

    J = helm3d.autograd.misfit(s2, solver, f, recv, data)
    J.backward()            # s2.grad = dJ/ds2 from the C ABI's adjoint solves

The forward pass refactors the solver for the given s2 (helm3d_set_medium)
and calls helm3d_misfit_grad, which returns the misfit and its gradient
together (forward and adjoint solves); backward scales the stored gradient.
"""
from __future__ import annotations

import torch


class Misfit(torch.autograd.Function):
    @staticmethod
    def forward(ctx, s2, solver, f, recv, data):
        solver.set_medium(s2.detach().contiguous())
        J, grad = solver.misfit_grad(f, recv, data)
        ctx.save_for_backward(grad)
        return torch.tensor(J, dtype=torch.float64, device=s2.device)

    @staticmethod
    def backward(ctx, gJ):
        (grad,) = ctx.saved_tensors
        return gJ * grad, None, None, None, None


def misfit(s2: torch.Tensor, solver, f: torch.Tensor, recv: torch.Tensor, data: torch.Tensor) -> torch.Tensor:
    """0.5 sum_s ||u_s[recv] - data_s||^2 as a differentiable function of s2."""
    return Misfit.apply(s2, solver, f, recv, data)
