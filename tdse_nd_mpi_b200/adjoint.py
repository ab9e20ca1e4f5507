"""PyTorch bridge to the engine's adjoint: dJ/dE of a length-gauge run.

``length_gauge_objective(grid, psi0, E, weight)`` returns J = dNr sum_x w(x) |psi_T(x)|^2 as a
torch scalar for the field samples E [nsteps, s, dim] (the F.E layout of integrators.c:81-101)
and, through ``torch.autograd``, its gradient with respect to E. Both come from one call of
``qnd_adjoint_length`` (the C ABI), which runs the forward steps keeping a state every
``checkpoint`` steps and then the adjoint state backward, recomputing the states in between; the
gradient is held for ``backward``. The reference has no counterpart (the differentiation
extension).
"""
from __future__ import annotations

import numpy as np
import torch

from .engine import Grid


class LengthGaugeObjective(torch.autograd.Function):
    @staticmethod
    def forward(ctx, E, grid: Grid, psi0, weight, checkpoint: int):
        J, grad = grid.adjoint_length(psi0, E.detach().to("cpu", torch.float64).numpy(), weight, checkpoint)
        ctx.save_for_backward(torch.as_tensor(grad, dtype=E.dtype, device=E.device))
        return torch.tensor(J, dtype=E.dtype, device=E.device)

    @staticmethod
    def backward(ctx, gJ):
        (g,) = ctx.saved_tensors
        return gJ * g, None, None, None, None


def length_gauge_objective(grid: Grid, psi0, E: torch.Tensor, weight, checkpoint: int = 50) -> torch.Tensor:
    return LengthGaugeObjective.apply(E, grid, psi0, weight, checkpoint)


def absorbed_weight(grid: Grid, radius: float) -> np.ndarray:
    """w = 1 where |r| > radius, 0 inside: J is then the norm beyond that radius."""
    X = np.meshgrid(*[grid.axis_r(j) for j in range(grid.dim)], indexing="ij")
    return (np.sqrt(sum(x * x for x in X)) > radius).astype(np.float64)
