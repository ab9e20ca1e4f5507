"""PyTorch bridge to the engine's adjoint: dJ/dE of a length-gauge run.

``length_gauge_objective(grid, psi0, E, weight)`` returns J = dNr sum_x w(x) |psi_T(x)|^2 as a
torch scalar for the field samples E [nsteps, s, dim] (the F.E layout of integrators.c:81-101)
and, through ``torch.autograd``, its gradient with respect to E; ``velocity_gauge_objective`` does
the same for the vector-potential samples A of a velocity-gauge run. J and its gradient come from
one call of ``qnd_adjoint_length`` or ``qnd_adjoint_velocity`` (the C ABI). That call runs the
forward steps keeping a state every ``checkpoint`` steps, then the adjoint state backward,
recomputing the states in between. The gradient is held for ``backward``. The reference has no counterpart (the differentiation
extension).
"""
from __future__ import annotations

import numpy as np
import torch

from .engine import Grid


class GaugeObjective(torch.autograd.Function):
    @staticmethod
    def forward(ctx, F, grid: Grid, psi0, weight, checkpoint: int, velocity: bool):
        run = grid.adjoint_velocity if velocity else grid.adjoint_length
        J, grad = run(psi0, F.detach().to("cpu", torch.float64).numpy(), weight, checkpoint)
        ctx.save_for_backward(torch.as_tensor(grad, dtype=F.dtype, device=F.device))
        return torch.tensor(J, dtype=F.dtype, device=F.device)

    @staticmethod
    def backward(ctx, gJ):
        (g,) = ctx.saved_tensors
        return gJ * g, None, None, None, None, None


def length_gauge_objective(grid: Grid, psi0, E: torch.Tensor, weight, checkpoint: int = 50) -> torch.Tensor:
    """J of a length-gauge run with field samples E; differentiable in E."""
    return GaugeObjective.apply(E, grid, psi0, weight, checkpoint, False)


def velocity_gauge_objective(grid: Grid, psi0, A: torch.Tensor, weight, checkpoint: int = 50) -> torch.Tensor:
    """J of a velocity-gauge run with vector-potential samples A; differentiable in A."""
    return GaugeObjective.apply(A, grid, psi0, weight, checkpoint, True)


def absorbed_weight(grid: Grid, radius: float) -> np.ndarray:
    """w = 1 where |r| > radius, 0 inside: J is then the norm beyond that radius."""
    X = np.meshgrid(*[grid.axis_r(j) for j in range(grid.dim)], indexing="ij")
    return (np.sqrt(sum(x * x for x in X)) > radius).astype(np.float64)
