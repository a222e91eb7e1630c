// PyTorch operators over the fresco_b200 potentials, registered with the
// dispatcher (torch.ops.fresco.*), so that a PyTorch program reaches the
// device evaluation as an operator: autograd, torch.compile graphs and the
// current CUDA stream work as for any other op.
//
//   fresco::energy(int potential, Tensor x) -> Tensor
//   fresco::energy_gradient(int potential, Tensor x) -> (Tensor, Tensor)
//       the reference's get_energy / get_energy_gradient
//       (fresco/potentials/*.pyx, base_potential.hpp:28-43) in the
//       potential's own gradient convention;
//   fresco::loss(int potential, Tensor x) -> (Tensor, Tensor)
//       energy and the exact derivative with respect to x (convention 1 of
//       fresco_potential_set_gradient_mode, restored afterwards); the Python
//       side registers its backward (grad_energy * gradient).
//
// `potential` is the address of a fresco_potential (the handle the Python
// objects hold); x is the flat float64 coordinate vector on a CUDA device.
// The work is enqueued on PyTorch's current stream of x's device.  Meta
// kernels give the output shapes to fake-tensor tracing.
#include <ATen/ATen.h>
#include <c10/cuda/CUDAGuard.h>
#include <c10/cuda/CUDAStream.h>
#include <torch/library.h>

#include <tuple>

#include "fresco_b200.h"

namespace {

fresco_potential as_potential(int64_t handle) {
  TORCH_CHECK_VALUE(handle != 0, "fresco: null potential handle");
  return reinterpret_cast<fresco_potential>(static_cast<intptr_t>(handle));
}

void check_x(const at::Tensor& x) {
  TORCH_CHECK_VALUE(x.is_cuda(), "fresco: x must be a CUDA tensor");
  TORCH_CHECK_VALUE(x.scalar_type() == at::kDouble, "fresco: x must be float64");
  TORCH_CHECK_VALUE(x.dim() == 1, "fresco: x must be the flat coordinate vector");
}

void check_rc(int rc) {
  if (rc == FRESCO_OK) return;
  if (rc == FRESCO_ERR_INVALID) TORCH_CHECK_VALUE(false, "fresco: ", fresco_last_error());
  TORCH_CHECK(false, "fresco: ", fresco_last_error());
}

void* current_stream(const at::Tensor& x) {
  return static_cast<void*>(c10::cuda::getCurrentCUDAStream(x.device().index()).stream());
}

at::Tensor energy_cuda(int64_t potential, const at::Tensor& x_in) {
  check_x(x_in);
  const at::Tensor x = x_in.contiguous();
  const c10::cuda::CUDAGuard guard(x.device());
  at::Tensor e = at::zeros({}, x.options());
  check_rc(fresco_potential_energy_device(as_potential(potential), x.data_ptr<double>(), x.numel(),
                                          e.data_ptr<double>(), 0, current_stream(x)));
  return e;
}

std::tuple<at::Tensor, at::Tensor> energy_gradient_cuda(int64_t potential, const at::Tensor& x_in) {
  check_x(x_in);
  const at::Tensor x = x_in.contiguous();
  const c10::cuda::CUDAGuard guard(x.device());
  at::Tensor e = at::zeros({}, x.options());
  at::Tensor g = at::empty_like(x);
  check_rc(fresco_potential_energy_gradient_device(as_potential(potential), x.data_ptr<double>(), x.numel(),
                                                   g.data_ptr<double>(), e.data_ptr<double>(), 0,
                                                   current_stream(x)));
  return {e, g};
}

std::tuple<at::Tensor, at::Tensor> loss_cuda(int64_t potential, const at::Tensor& x) {
  check_x(x);  // before the handle is touched
  fresco_potential p = as_potential(potential);
  int prev = 0;
  check_rc(fresco_potential_gradient_mode(p, &prev));
  check_rc(fresco_potential_set_gradient_mode(p, 1));
  std::tuple<at::Tensor, at::Tensor> out;
  try {
    out = energy_gradient_cuda(potential, x);
  } catch (...) {
    fresco_potential_set_gradient_mode(p, prev);
    throw;
  }
  check_rc(fresco_potential_set_gradient_mode(p, prev));
  return out;
}

at::Tensor energy_meta(int64_t, const at::Tensor& x) { return at::empty({}, x.options()); }

std::tuple<at::Tensor, at::Tensor> energy_gradient_meta(int64_t, const at::Tensor& x) {
  return {at::empty({}, x.options()), at::empty_like(x)};
}

}  // namespace

TORCH_LIBRARY(fresco, m) {
  m.def("energy(int potential, Tensor x) -> Tensor");
  m.def("energy_gradient(int potential, Tensor x) -> (Tensor, Tensor)");
  m.def("loss(int potential, Tensor x) -> (Tensor, Tensor)");
}

TORCH_LIBRARY_IMPL(fresco, CUDA, m) {
  m.impl("energy", energy_cuda);
  m.impl("energy_gradient", energy_gradient_cuda);
  m.impl("loss", loss_cuda);
}

// CPU tensors reach the same functions, which reject them with a ValueError
TORCH_LIBRARY_IMPL(fresco, CPU, m) {
  m.impl("energy", energy_cuda);
  m.impl("energy_gradient", energy_gradient_cuda);
  m.impl("loss", loss_cuda);
}

TORCH_LIBRARY_IMPL(fresco, Meta, m) {
  m.impl("energy", energy_meta);
  m.impl("energy_gradient", energy_gradient_meta);
  m.impl("loss", energy_gradient_meta);
}
