"""PyTorch operators over the potentials (torch.ops.fresco.*) on the device: the same results as the
C-ABI calls, the registered backward of fresco::loss (the exact gradient), PyTorch's current stream,
torch.compile tracing, and argument errors."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _pot(prec="fp64"):
    from fresco_b200 import NUwU

    x, radii, Sk, V, L = O.stealthy_nuwu_inputs(1500, 12, 8, ndim=2, seed=4)
    radii = 0.5 + np.random.default_rng(1).random(1500)
    return NUwU(radii, 12, Sk, V, L, eps=1e-12 if prec == "fp64" else 1e-6, precision=prec), x


def test_energy_and_energy_gradient_match_the_potential():
    import torch

    from fresco_b200 import ops

    pot, x = _pot()
    e_ref, g_ref = pot.get_energy_gradient(x)
    xt = torch.tensor(x, device="cuda")
    e, g = ops.energy_gradient(pot, xt)
    assert abs(float(e) - e_ref) <= 1e-13 * abs(e_ref)
    assert np.allclose(g.cpu().numpy(), g_ref, rtol=1e-12, atol=1e-12 * np.abs(g_ref).max())
    assert abs(float(ops.energy(pot, xt)) - e_ref) <= 1e-13 * abs(e_ref)


def test_loss_backward_is_the_exact_gradient_and_keeps_the_mode():
    import torch

    from fresco_b200 import ops

    pot, x = _pot()
    _, g_reference = pot.get_energy_gradient(x)
    pot.set_gradient_mode("exact")
    e_ref, g_exact = pot.get_energy_gradient(x)
    pot.set_gradient_mode("reference")
    xt = torch.tensor(x, device="cuda", requires_grad=True)
    total = 2.0 * ops.loss(pot, xt) + (xt ** 2).sum()
    total.backward()
    want = 2.0 * g_exact + 2.0 * x
    assert np.allclose(xt.grad.cpu().numpy(), want, rtol=1e-12, atol=1e-12 * np.abs(want).max())
    assert pot.gradient_mode() == "reference"
    _, g_after = pot.get_energy_gradient(x)  # the handle is back in the reference convention
    assert np.allclose(g_after, g_reference, rtol=1e-12, atol=1e-12 * np.abs(g_reference).max())


def test_current_stream_and_compile():
    import torch

    from fresco_b200 import ops

    pot, x = _pot("fp32")
    h = ops.handle_of(pot)
    xt = torch.tensor(x, device="cuda")
    e0, g0 = torch.ops.fresco.loss(h, xt)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        e1, g1 = torch.ops.fresco.loss(h, xt)
    s.synchronize()
    assert float(e1) == pytest.approx(float(e0), rel=1e-6)

    def f(y):
        e, g = torch.ops.fresco.loss(h, y)
        return 3.0 * e + g.square().sum()

    fc = torch.compile(f, backend="aot_eager", fullgraph=True)
    y = xt.clone().requires_grad_(True)
    out = fc(y)
    assert float(out) == pytest.approx(float(f(xt)), rel=1e-6)
    out.backward()
    assert torch.allclose(y.grad, 3.0 * g0, rtol=1e-5, atol=1e-5 * float(g0.abs().max()))


def test_argument_errors():
    import torch

    from fresco_b200 import ops

    pot, x = _pot()
    with pytest.raises(ValueError, match="CUDA"):
        ops.energy_gradient(pot, torch.tensor(x))
    with pytest.raises(ValueError, match="float64"):
        ops.energy_gradient(pot, torch.tensor(x, device="cuda", dtype=torch.float32))
    with pytest.raises(ValueError):
        ops.energy_gradient(pot, torch.tensor(x[:-2], device="cuda"))  # wrong coordinate count
