"""The PyTorch operator library (fresco_b200/libfresco_torch.so, csrc/torch_ops.cpp) on CPU: it loads,
registers fresco::energy / energy_gradient / loss with the dispatcher, and its meta kernels give
fake-tensor tracing the output shapes.  The CUDA kernels are tested in test_torch_ops_gpu.py."""
import torch


def test_operators_registered():
    from fresco_b200 import ops  # noqa: F401

    schemas = {n: str(getattr(torch.ops.fresco, n).default._schema) for n in ("energy", "energy_gradient", "loss")}
    assert schemas["energy"] == "fresco::energy(int potential, Tensor x) -> Tensor"
    assert schemas["energy_gradient"] == "fresco::energy_gradient(int potential, Tensor x) -> (Tensor, Tensor)"
    assert schemas["loss"] == "fresco::loss(int potential, Tensor x) -> (Tensor, Tensor)"


def test_meta_shapes_under_fake_tensors():
    from torch._subclasses.fake_tensor import FakeTensorMode

    from fresco_b200 import ops  # noqa: F401

    with FakeTensorMode():
        x = torch.empty(2 * 4096, dtype=torch.float64, device="cuda")
        e = torch.ops.fresco.energy(1, x)
        e2, g = torch.ops.fresco.energy_gradient(1, x)
        e3, g3 = torch.ops.fresco.loss(1, x)
    assert e.shape == e2.shape == e3.shape == torch.Size([])
    assert g.shape == g3.shape == x.shape and g.dtype == torch.float64


def test_cpu_tensors_are_refused():
    import pytest

    from fresco_b200 import ops  # noqa: F401

    x = torch.zeros(8, dtype=torch.float64)
    for op in (torch.ops.fresco.energy, torch.ops.fresco.energy_gradient, torch.ops.fresco.loss):
        with pytest.raises(ValueError, match="CUDA"):
            op(1, x)
