// PyTorch operator library over the C ABI: torch.ops.dnsbox.*.
//
// The operators take a context handle (the dnsbox_ctx pointer as an int,
// Box.handle on the Python side) and CUDA tensors in the library's layouts,
// run on torch's current CUDA stream of the tensor's device, and allocate
// their outputs through the caching allocator.  They are registered for the
// CUDA dispatch key only: there is no CPU path.  The reference's operator
// surface they expose: rhs_nonlinear (rhs.f90:18-135), the transpose of its
// linearisation (the exact counterpart of rhsAdj.f90's rhsNonlinearAdj),
// the time step (dnsboxheun.f90:85-126 / dnsbox.f90:87-218 /
// dnsboximplicit.f90:88-181), the residual J and its gradient
// (rhsupptilde, rhsAdj.f90:177-213) and p3dfft's transforms (state.f90:58-72).
#include <ATen/ATen.h>
#include <c10/cuda/CUDAGuard.h>
#include <c10/cuda/CUDAStream.h>
#include <torch/library.h>

#include <string>
#include <tuple>

#include "../../include/dnsbox.h"

namespace {

dnsbox_ctx *ctx_of(int64_t h) {
  TORCH_CHECK(h != 0, "dnsbox: null context handle");
  return reinterpret_cast<dnsbox_ctx *>(static_cast<intptr_t>(h));
}

void check(int rc, const char *what) {
  TORCH_CHECK(rc == DNSBOX_OK, "dnsbox ", what, " failed (", rc, "): ", dnsbox_last_error());
}

// Binds the context to the current stream of the tensor's device.
dnsbox_ctx *bind(int64_t h, const at::Tensor &t) {
  TORCH_CHECK(t.is_cuda() && t.is_contiguous(), "dnsbox: tensors must be contiguous CUDA tensors");
  dnsbox_ctx *c = ctx_of(h);
  check(dnsbox_set_stream(c, c10::cuda::getCurrentCUDAStream(t.device().index()).stream()), "set_stream");
  return c;
}

at::Tensor rhs_nonlinear(int64_t h, const at::Tensor &uh) {
  c10::cuda::CUDAGuard g(uh.device());
  dnsbox_ctx *c = bind(h, uh);
  at::Tensor out = at::empty_like(uh);
  check(dnsbox_rhs_nonlinear(c, uh.data_ptr(), out.data_ptr(), nullptr), "rhs_nonlinear");
  return out;
}

at::Tensor rhs_nonlinear_vjp(int64_t h, const at::Tensor &uh, const at::Tensor &gout) {
  c10::cuda::CUDAGuard g(uh.device());
  dnsbox_ctx *c = bind(h, uh);
  at::Tensor gc = gout.contiguous();
  at::Tensor out = at::empty_like(uh);
  check(dnsbox_rhs_nonlinear_vjp(c, uh.data_ptr(), gc.data_ptr(), out.data_ptr()), "rhs_nonlinear_vjp");
  return out;
}

void step_(int64_t h, at::Tensor &uh, int64_t nsteps) {
  c10::cuda::CUDAGuard g(uh.device());
  dnsbox_ctx *c = bind(h, uh);
  check(dnsbox_step(c, uh.data_ptr(), (int)nsteps, nullptr), "step");
}

std::tuple<at::Tensor, at::Tensor> residual_grad(int64_t h, const at::Tensor &uh) {
  c10::cuda::CUDAGuard g(uh.device());
  dnsbox_ctx *c = bind(h, uh);
  at::Tensor grad = at::empty_like(uh);
  double J = 0.0;
  check(dnsbox_residual_grad(c, uh.data_ptr(), grad.data_ptr(), &J), "residual_grad");
  return {at::full({}, J, uh.options().dtype(at::kDouble)), grad};
}

at::Tensor residual(int64_t h, const at::Tensor &uh) {
  c10::cuda::CUDAGuard g(uh.device());
  dnsbox_ctx *c = bind(h, uh);
  double J = 0.0;
  check(dnsbox_residual(c, uh.data_ptr(), &J), "residual");
  return at::full({}, J, uh.options().dtype(at::kDouble));
}

at::Tensor c2r(int64_t h, const at::Tensor &spec, int64_t nx) {
  c10::cuda::CUDAGuard g(spec.device());
  dnsbox_ctx *c = bind(h, spec);
  auto sizes = spec.sizes().vec();
  sizes.back() = nx;
  at::Tensor out = at::empty(sizes, spec.options().dtype(spec.scalar_type() == at::kComplexDouble ? at::kDouble
                                                                                                  : at::kFloat));
  check(dnsbox_c2r(c, spec.data_ptr(), out.data_ptr()), "c2r");
  return out;
}

at::Tensor r2c(int64_t h, const at::Tensor &phys) {
  c10::cuda::CUDAGuard g(phys.device());
  dnsbox_ctx *c = bind(h, phys);
  auto sizes = phys.sizes().vec();
  sizes.back() = sizes.back() / 2 + 1;
  at::Tensor out = at::empty(sizes, phys.options().dtype(phys.scalar_type() == at::kDouble ? at::kComplexDouble
                                                                                           : at::kComplexFloat));
  check(dnsbox_r2c(c, phys.data_ptr(), out.data_ptr()), "r2c");
  return out;
}

}  // namespace

TORCH_LIBRARY(dnsbox, m) {
  m.def("rhs_nonlinear(int ctx, Tensor uhat) -> Tensor");
  m.def("rhs_nonlinear_vjp(int ctx, Tensor uhat, Tensor g) -> Tensor");
  m.def("step_(int ctx, Tensor(a!) uhat, int nsteps) -> ()");
  m.def("residual(int ctx, Tensor uhat) -> Tensor");
  m.def("residual_grad(int ctx, Tensor uhat) -> (Tensor, Tensor)");
  m.def("c2r(int ctx, Tensor spec, int nx) -> Tensor");
  m.def("r2c(int ctx, Tensor phys) -> Tensor");
}

TORCH_LIBRARY_IMPL(dnsbox, CUDA, m) {
  m.impl("rhs_nonlinear", &rhs_nonlinear);
  m.impl("rhs_nonlinear_vjp", &rhs_nonlinear_vjp);
  m.impl("step_", &step_);
  m.impl("residual", &residual);
  m.impl("residual_grad", &residual_grad);
  m.impl("c2r", &c2r);
  m.impl("r2c", &r2c);
}
