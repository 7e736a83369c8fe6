// XLA FFI handlers over the C ABI of include/rfxb200.h: the drop-in for the
// body of rfx's lax.scan (rfx/simulation.py:1958-1977, called from
// Simulation.forward through rfx/api/_execute.py:1534) when the caller is a
// jax.jit-ed program.  Built only where jaxlib's FFI headers exist
// (jax.ffi.include_dir()); rfx_b200/build.py compiles it into
// rfx_b200/librfxb200_ffi.so linked against librfxb200.so.
//
// A plan (rfxb_plan_create) is created by the Python side before tracing and
// passed as the int64 attribute "plan"; it owns the padded state, CPML psi,
// the gradient-region history and the adjoint state.  XLA owns every buffer
// below and passes its compute stream.  The handlers:
//
//   rfxb_ffi_forward          eps_r, sigma, source table -> probe traces and
//                             the final six fields (state reset first: a run
//                             from rest, as run() / forward() start)
//   rfxb_ffi_forward_record   the same, recording the gradient region's
//                             history for rfxb_ffi_adjoint (the forward half
//                             of a jax.custom_vjp)
//   rfxb_ffi_adjoint          probe cotangents, d ca/d eps_r and d cb/d eps_r
//                             over the region -> dJ/d eps_r over the region
//                             (float64) and dJ/d source table (the backward
//                             half; replaces jax.grad through the scan)
//
// Errors come back as ffi::Error(kInternal, rfxb_last_error()); nothing is
// raised inside kernels.
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "rfxb200.h"
#include "xla/ffi/api/ffi.h"

namespace ffi = xla::ffi;

namespace {

ffi::Error fail(const char* what, int rc) {
  return ffi::Error(ffi::ErrorCode::kInternal,
                    std::string(what) + " failed (" + std::to_string(rc) + "): " + rfxb_last_error());
}

RfxbPlan* as_plan(int64_t p) { return reinterpret_cast<RfxbPlan*>(static_cast<intptr_t>(p)); }

ffi::Error run_forward(cudaStream_t st, int64_t plan, int64_t n_steps, bool record, ffi::Buffer<ffi::F32> eps,
                       ffi::Buffer<ffi::F32> sigma, ffi::Buffer<ffi::F32> src, ffi::ResultBuffer<ffi::F32> probes,
                       ffi::ResultBuffer<ffi::F32> ex, ffi::ResultBuffer<ffi::F32> ey,
                       ffi::ResultBuffer<ffi::F32> ez, ffi::ResultBuffer<ffi::F32> hx,
                       ffi::ResultBuffer<ffi::F32> hy, ffi::ResultBuffer<ffi::F32> hz) {
  RfxbPlan* p = as_plan(plan);
  if (!p) return ffi::Error(ffi::ErrorCode::kInvalidArgument, "rfxb FFI: null plan attribute");
  int rc = rfxb_plan_set_materials(p, eps.typed_data(), sigma.typed_data(), nullptr, nullptr, st);
  if (rc) return fail("rfxb_plan_set_materials", rc);
  if ((rc = rfxb_plan_reset(p, st))) return fail("rfxb_plan_reset", rc);
  if (record && (rc = rfxb_plan_record_history(p, 0, static_cast<int>(n_steps))))
    return fail("rfxb_plan_record_history", rc);
  RfxbStepIO io{};
  io.src_wave_dev = src.element_count() ? src.typed_data() : nullptr;
  io.probe_out_dev = probes->element_count() ? probes->typed_data() : nullptr;
  if ((rc = rfxb_plan_advance(p, &io, 0, static_cast<int>(n_steps), st))) return fail("rfxb_plan_advance", rc);
  float* f[6] = {ex->typed_data(), ey->typed_data(), ez->typed_data(),
                 hx->typed_data(), hy->typed_data(), hz->typed_data()};
  if ((rc = rfxb_plan_store_fields(p, f, st))) return fail("rfxb_plan_store_fields", rc);
  return ffi::Error::Success();
}

ffi::Error Forward(cudaStream_t st, int64_t plan, int64_t n_steps, ffi::Buffer<ffi::F32> eps,
                   ffi::Buffer<ffi::F32> sigma, ffi::Buffer<ffi::F32> src, ffi::ResultBuffer<ffi::F32> probes,
                   ffi::ResultBuffer<ffi::F32> ex, ffi::ResultBuffer<ffi::F32> ey, ffi::ResultBuffer<ffi::F32> ez,
                   ffi::ResultBuffer<ffi::F32> hx, ffi::ResultBuffer<ffi::F32> hy, ffi::ResultBuffer<ffi::F32> hz) {
  return run_forward(st, plan, n_steps, false, eps, sigma, src, probes, ex, ey, ez, hx, hy, hz);
}

ffi::Error ForwardRecord(cudaStream_t st, int64_t plan, int64_t n_steps, ffi::Buffer<ffi::F32> eps,
                         ffi::Buffer<ffi::F32> sigma, ffi::Buffer<ffi::F32> src, ffi::ResultBuffer<ffi::F32> probes,
                         ffi::ResultBuffer<ffi::F32> ex, ffi::ResultBuffer<ffi::F32> ey,
                         ffi::ResultBuffer<ffi::F32> ez, ffi::ResultBuffer<ffi::F32> hx,
                         ffi::ResultBuffer<ffi::F32> hy, ffi::ResultBuffer<ffi::F32> hz) {
  return run_forward(st, plan, n_steps, true, eps, sigma, src, probes, ex, ey, ez, hx, hy, hz);
}

ffi::Error Adjoint(cudaStream_t st, int64_t plan, int64_t n_steps, ffi::Buffer<ffi::F32> g,
                   ffi::Buffer<ffi::F32> dca, ffi::Buffer<ffi::F32> dcb, ffi::ResultBuffer<ffi::F64> grad,
                   ffi::ResultBuffer<ffi::F32> src_adj) {
  RfxbPlan* p = as_plan(plan);
  if (!p) return ffi::Error(ffi::ErrorCode::kInvalidArgument, "rfxb FFI: null plan attribute");
  if (cudaMemsetAsync(grad->typed_data(), 0, grad->element_count() * sizeof(double), st) != cudaSuccess ||
      (src_adj->element_count() &&
       cudaMemsetAsync(src_adj->typed_data(), 0, src_adj->element_count() * sizeof(float), st) != cudaSuccess))
    return ffi::Error(ffi::ErrorCode::kInternal, "rfxb FFI: clearing the gradient outputs failed");
  RfxbAdjointIO a{};
  a.g_dev = g.typed_data();
  a.grad_dev = grad->typed_data();
  a.dca_dev = dca.typed_data();
  a.dcb_dev = dcb.typed_data();
  a.src_adj_dev = src_adj->element_count() ? src_adj->typed_data() : nullptr;
  const int n = static_cast<int>(n_steps);
  int rc = rfxb_plan_adjoint_begin(p, &a, n, st);
  if (rc) return fail("rfxb_plan_adjoint_begin", rc);
  if ((rc = rfxb_plan_adjoint_advance(p, &a, n, n, st))) return fail("rfxb_plan_adjoint_advance", rc);
  return ffi::Error::Success();
}

}  // namespace

#define RFXB_FWD_BINDING                                       \
  ffi::Ffi::Bind()                                             \
      .Ctx<ffi::PlatformStream<cudaStream_t>>()                \
      .Attr<int64_t>("plan")                                   \
      .Attr<int64_t>("n_steps")                                \
      .Arg<ffi::Buffer<ffi::F32>>()  /* eps_r (nx, ny, nz) */   \
      .Arg<ffi::Buffer<ffi::F32>>()  /* sigma */                \
      .Arg<ffi::Buffer<ffi::F32>>()  /* source table (N, n_src) */ \
      .Ret<ffi::Buffer<ffi::F32>>()  /* probes (N, n_probe) */  \
      .Ret<ffi::Buffer<ffi::F32>>()                            \
      .Ret<ffi::Buffer<ffi::F32>>()                            \
      .Ret<ffi::Buffer<ffi::F32>>()                            \
      .Ret<ffi::Buffer<ffi::F32>>()                            \
      .Ret<ffi::Buffer<ffi::F32>>()                            \
      .Ret<ffi::Buffer<ffi::F32>>()

XLA_FFI_DEFINE_HANDLER_SYMBOL(RfxbFfiForward, Forward, RFXB_FWD_BINDING);
XLA_FFI_DEFINE_HANDLER_SYMBOL(RfxbFfiForwardRecord, ForwardRecord, RFXB_FWD_BINDING);
XLA_FFI_DEFINE_HANDLER_SYMBOL(RfxbFfiAdjoint, Adjoint,
                              ffi::Ffi::Bind()
                                  .Ctx<ffi::PlatformStream<cudaStream_t>>()
                                  .Attr<int64_t>("plan")
                                  .Attr<int64_t>("n_steps")
                                  .Arg<ffi::Buffer<ffi::F32>>()   // probe cotangents (N, n_probe)
                                  .Arg<ffi::Buffer<ffi::F32>>()   // d ca / d eps_r over the region
                                  .Arg<ffi::Buffer<ffi::F32>>()   // d cb / d eps_r over the region
                                  .Ret<ffi::Buffer<ffi::F64>>()   // dJ/d eps_r over the region
                                  .Ret<ffi::Buffer<ffi::F32>>()); // dJ/d source table (N, n_src)
