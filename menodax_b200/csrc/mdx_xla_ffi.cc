// XLA FFI handlers over the C ABI: the JAX front end's custom calls.
//
// Replaces the reference's generic launcher modax_numba_cuda_abi_launch
// (modax/_jax_numba_custom_call.py:145-231), which took a CUfunction, a launch
// shape and an argument-kind list as attributes.  Here the attributes name a
// plan (an mdx_plan* created by mdx_plan_create and kept alive by the Python
// side for the life of the process, as the reference keeps its CUfunction) and
// the solver's scalars; the buffers are XLA's, row-major, in the C ABI's order.
//
//   mdx_xla_solve: y0 (N, n_system) f64, times (S,) f64, params (N, P) f64,
//                  weights (N, n_system) f64 or (0,)
//               -> hist (N, S_hist, n_system) f64, counters (4, N) s32,
//                  workspace u8 (the persistent launch's queue head),
//                  ckpt f64 and ckpt_count (N,) s32 (a checkpointing plan; else (1,))
//   mdx_xla_grad:  times, params, ckpt, ckpt_count, grad_hist (N, S, n) f64,
//                  order (N,) s32
//               -> grad_y0 (N, n) f64, grad_params (N, P) f64, status (N,) s32
//
// Errors come back as ffi::Error with mdx_last_error's message.  Built only
// where JAX's FFI headers exist (jax.ffi.include_dir()), into
// libmenodax_b200_xla.so linked against libmenodax_b200.so.
#include <cuda_runtime_api.h>

#include <cstdint>
#include <string>

#include "../../include/menodax.h"
#include "xla/ffi/api/ffi.h"

namespace ffi = xla::ffi;

namespace {

ffi::Error last_error(const char* what) {
  char msg[2048];
  mdx_last_error(msg, sizeof msg);
  return ffi::Error(ffi::ErrorCode::kInternal, std::string(what) + ": " + msg);
}

ffi::Error MdxXlaSolve(cudaStream_t stream, int64_t plan, int32_t mode, double dt0, double rtol, double atol,
                       int32_t max_steps, int64_t ckpt_capacity, ffi::Buffer<ffi::F64> y0,
                       ffi::Buffer<ffi::F64> times, ffi::Buffer<ffi::F64> params, ffi::Buffer<ffi::F64> weights,
                       ffi::ResultBuffer<ffi::F64> hist, ffi::ResultBuffer<ffi::S32> counters,
                       ffi::ResultBuffer<ffi::U8> workspace, ffi::ResultBuffer<ffi::F64> ckpt,
                       ffi::ResultBuffer<ffi::S32> ckpt_count) {
  const auto y0_dims = y0.dimensions();
  const auto hist_dims = hist->dimensions();
  if (y0_dims.size() != 2 || hist_dims.size() != 3)
    return ffi::Error(ffi::ErrorCode::kInvalidArgument, "mdx_xla_solve: y0 must be 2-D and hist 3-D");
  const int64_t n = y0_dims[0];
  mdx_solve_desc d = {};
  d.struct_size = sizeof(d);
  d.mode = mode;
  d.n_traj = (int)n;
  d.n_save = (int)times.element_count();
  d.n_save_hist = (int)hist_dims[1];
  d.max_steps = max_steps;
  d.dt0 = dt0;
  d.rtol = rtol;
  d.atol = atol;
  d.y0 = y0.typed_data();
  d.times = times.typed_data();
  d.params = params.element_count() ? params.typed_data() : nullptr;
  d.weights = weights.element_count() ? weights.typed_data() : nullptr;
  d.hist = hist->typed_data();
  int32_t* c = counters->typed_data();
  d.accepted = c;
  d.rejected = c + n;
  d.loop_steps = c + 2 * n;
  d.status = c + 3 * n;
  d.workspace = workspace->typed_data();
  d.workspace_bytes = workspace->size_bytes();
  if (ckpt_capacity > 0) {
    d.ckpt = ckpt->typed_data();
    d.ckpt_count = ckpt_count->typed_data();
    d.ckpt_capacity = ckpt_capacity;
  }
  if (mdx_solve(reinterpret_cast<mdx_plan*>(plan), &d, stream) != MDX_OK) return last_error("mdx_solve");
  return ffi::Error::Success();
}

ffi::Error MdxXlaGrad(cudaStream_t stream, int64_t plan, int64_t ckpt_capacity, ffi::Buffer<ffi::F64> times,
                      ffi::Buffer<ffi::F64> params, ffi::Buffer<ffi::F64> ckpt, ffi::Buffer<ffi::S32> ckpt_count,
                      ffi::Buffer<ffi::F64> grad_hist, ffi::Buffer<ffi::S32> order,
                      ffi::ResultBuffer<ffi::F64> grad_y0, ffi::ResultBuffer<ffi::F64> grad_params,
                      ffi::ResultBuffer<ffi::S32> status) {
  mdx_grad_desc d = {};
  d.struct_size = sizeof(d);
  d.n_traj = (int)ckpt_count.element_count();
  d.n_save = (int)times.element_count();
  d.times = times.typed_data();
  d.params = params.element_count() ? params.typed_data() : nullptr;
  d.ckpt = ckpt.typed_data();
  d.ckpt_count = ckpt_count.typed_data();
  d.ckpt_capacity = ckpt_capacity;
  d.grad_hist = grad_hist.typed_data();
  d.grad_y0 = grad_y0->typed_data();
  d.grad_params = grad_params->typed_data();
  d.status = status->typed_data();
  d.order = order.typed_data();
  if (mdx_grad(reinterpret_cast<mdx_plan*>(plan), &d, stream) != MDX_OK) return last_error("mdx_grad");
  return ffi::Error::Success();
}

}  // namespace

XLA_FFI_DEFINE_HANDLER_SYMBOL(mdx_xla_solve, MdxXlaSolve,
                              ffi::Ffi::Bind()
                                  .Ctx<ffi::PlatformStream<cudaStream_t>>()
                                  .Attr<int64_t>("plan")
                                  .Attr<int32_t>("mode")
                                  .Attr<double>("dt0")
                                  .Attr<double>("rtol")
                                  .Attr<double>("atol")
                                  .Attr<int32_t>("max_steps")
                                  .Attr<int64_t>("ckpt_capacity")
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Ret<ffi::Buffer<ffi::F64>>()
                                  .Ret<ffi::Buffer<ffi::S32>>()
                                  .Ret<ffi::Buffer<ffi::U8>>()
                                  .Ret<ffi::Buffer<ffi::F64>>()
                                  .Ret<ffi::Buffer<ffi::S32>>());

XLA_FFI_DEFINE_HANDLER_SYMBOL(mdx_xla_grad, MdxXlaGrad,
                              ffi::Ffi::Bind()
                                  .Ctx<ffi::PlatformStream<cudaStream_t>>()
                                  .Attr<int64_t>("plan")
                                  .Attr<int64_t>("ckpt_capacity")
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Arg<ffi::Buffer<ffi::S32>>()
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Arg<ffi::Buffer<ffi::S32>>()
                                  .Ret<ffi::Buffer<ffi::F64>>()
                                  .Ret<ffi::Buffer<ffi::F64>>()
                                  .Ret<ffi::Buffer<ffi::S32>>());
