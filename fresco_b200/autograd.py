"""Differentiable structure-factor losses for PyTorch.

``structure_factor_loss(potential, x)`` returns the energy of any fresco_b200
potential as a 0-d CUDA tensor whose backward pass is the hand-written
adjoint computed on the device (for NUwU: the type-2 interpolation of
i k w (S - S0) rho; nuwu.hpp:260-315).  The forward call evaluates energy
and gradient together with the potential in its *exact* gradient mode, i.e.
the true derivative with respect to ``x`` (the reference's own formulas are
scaled differently, see ``BasePotential.set_gradient_mode``), so the result
composes with other autograd terms and passes finite-difference checks.

    x = torch.tensor(x0, device="cuda", requires_grad=True)
    e = structure_factor_loss(pot, x) + other_terms(x)
    e.backward()
"""
from __future__ import annotations

import torch

__all__ = ["StructureFactorLoss", "structure_factor_loss"]


class StructureFactorLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, potential):
        if not x.is_cuda or x.dtype != torch.float64:
            raise ValueError("x must be a float64 CUDA tensor")
        xd = x.detach().contiguous()
        prev = potential.gradient_mode()
        potential.set_gradient_mode("exact")
        try:
            e, g = potential.energy_gradient_device(xd)
        finally:
            potential.set_gradient_mode(prev)
        ctx.save_for_backward(g)
        return e

    @staticmethod
    def backward(ctx, grad_out):
        (g,) = ctx.saved_tensors
        return grad_out * g.view_as(g), None


def structure_factor_loss(potential, x):
    """Energy of ``potential`` at ``x`` (float64 CUDA tensor) with a device adjoint for backward."""
    return StructureFactorLoss.apply(x, potential)
