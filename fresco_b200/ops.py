"""PyTorch operators over fresco_b200 potentials.

Importing this module loads ``libfresco_torch.so`` (``csrc/torch_ops.cpp``, built next to the
CUDA library) and so registers three operators with the PyTorch dispatcher:

* ``torch.ops.fresco.energy(potential, x) -> energy``
* ``torch.ops.fresco.energy_gradient(potential, x) -> (energy, gradient)``: the reference's
  ``get_energy`` / ``get_energy_gradient`` (fresco/potentials/*.pyx) in the potential's own
  gradient convention;
* ``torch.ops.fresco.loss(potential, x) -> (energy, gradient)``: the gradient is the exact
  derivative with respect to ``x``, and autograd knows it: ``loss(p, x)[0].backward()`` gives
  ``x.grad = gradient``.

``potential`` is the integer handle of a fresco_b200 potential (``handle_of(pot)``), ``x`` the
flat float64 coordinates on a CUDA device; the evaluation is enqueued on PyTorch's current stream.
The operators have meta kernels, so fake-tensor tracing (``torch.compile``) sees their shapes.
"""
from __future__ import annotations

import ctypes as C
import os

import torch

__all__ = ["handle_of", "energy", "energy_gradient", "loss"]

_LIB = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libfresco_torch.so")
if not os.path.exists(_LIB):
    raise ImportError(f"fresco_b200: {_LIB} is not built (run fresco_b200/build.py)")

from . import _lib  # noqa: E402,F401  (loads libfresco_b200.so first)

torch.ops.load_library(_LIB)


def handle_of(potential) -> int:
    """The integer handle the operators take for a fresco_b200 potential (or an int handle)."""
    if isinstance(potential, int):
        return potential
    h = C.cast(potential.handle, C.c_void_p).value
    if not h:
        raise ValueError("the potential has no live handle")
    return int(h)


def _loss_setup_context(ctx, inputs, output):
    ctx.save_for_backward(output[1])


def _loss_backward(ctx, grad_energy, grad_gradient):
    (g,) = ctx.saved_tensors
    return None, grad_energy * g  # (potential, x); the gradient output is not differentiated


torch.library.register_autograd("fresco::loss", _loss_backward, setup_context=_loss_setup_context)


def energy(potential, x):
    return torch.ops.fresco.energy(handle_of(potential), x)


def energy_gradient(potential, x):
    return torch.ops.fresco.energy_gradient(handle_of(potential), x)


def loss(potential, x):
    """Energy (0-d tensor) of ``potential`` at ``x`` whose backward is the device adjoint."""
    return torch.ops.fresco.loss(handle_of(potential), x)[0]
