"""Differentiable structure-factor losses for PyTorch.

``structure_factor_loss(potential, x)`` returns the energy of any fresco_b200
potential as a 0-d CUDA tensor whose backward pass is the hand-written
adjoint computed on the device (for NUwU: the type-2 interpolation of
i k w (S - S0) rho; nuwu.hpp:260-315).  It is the registered operator
``torch.ops.fresco.loss`` (``fresco_b200.ops``): the forward call evaluates
energy and gradient together in the potential's *exact* gradient convention,
i.e. the true derivative with respect to ``x`` (the reference's own formulas
are scaled differently, see ``BasePotential.set_gradient_mode``), so the
result composes with other autograd terms, passes finite-difference checks
and can be traced by ``torch.compile``.

    x = torch.tensor(x0, device="cuda", requires_grad=True)
    e = structure_factor_loss(pot, x) + other_terms(x)
    e.backward()
"""
from __future__ import annotations

from . import ops

__all__ = ["StructureFactorLoss", "structure_factor_loss"]


def structure_factor_loss(potential, x):
    """Energy of ``potential`` at ``x`` (float64 CUDA tensor) with a device adjoint for backward."""
    if not x.is_cuda:
        raise ValueError("x must be a float64 CUDA tensor")
    return ops.loss(potential, x)


class StructureFactorLoss:
    """``StructureFactorLoss.apply(x, potential)``: the same as ``structure_factor_loss(potential, x)``."""

    @staticmethod
    def apply(x, potential):
        return structure_factor_loss(potential, x)
