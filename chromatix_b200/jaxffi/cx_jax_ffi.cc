// XLA FFI handlers over the C ABI (include/cx_b200.h), for the jax.ffi route
// into the library: the reference's functions are traced JAX code, so a
// chromatix build that dispatches its hot path here registers these handlers
// as CUDA custom-call targets (chromatix_b200/jaxffi/__init__.py does).
//
// Built only where jax is installed (its FFI headers come with jaxlib:
// jax.ffi.include_dir()); linked against libcx_b200.so.
//
//   cx_prop2d_ffi   Fourier-multiplier propagation (transfer / ASM): the
//                   FFT branch of kernel_propagate (functional/propagation.py:
//                   391-394) as reached from transfer_propagate / asm_propagate
//                   (:168-352).  Attribute conj_kernel = 1 gives the adjoint
//                   used by the custom_vjp backward.
#include <cuda_runtime.h>

#include <cstdint>

#include "cx_b200.h"
#include "xla/ffi/api/ffi.h"

namespace ffi = xla::ffi;

static ffi::Error Prop2D(cudaStream_t stream, ffi::Buffer<ffi::C64> u, ffi::Buffer<ffi::U8> planes,
                         ffi::ResultBuffer<ffi::C64> out, ffi::ResultBuffer<ffi::U8> workspace, int32_t ny,
                         int32_t nx, int32_t pad_y, int32_t pad_x, int32_t crop_y, int32_t crop_x, int32_t mode_same,
                         int32_t kernel, int32_t precision, int32_t remove_evanescent, int32_t bandlimit,
                         int32_t conj_kernel, double n_medium, double ky0, double kx0) {
  cx_prop2d_desc d{};
  d.ny = ny;
  d.nx = nx;
  d.pad_y = pad_y;
  d.pad_x = pad_x;
  d.n_wv = 1;
  d.n_in_planes = (int32_t)(u.element_count() / ((int64_t)ny * nx));
  d.n_out_planes = (int32_t)(planes.element_count() / sizeof(cx_plane));
  d.mode_same = mode_same;
  d.kernel = kernel;
  d.precision = precision;
  d.remove_evanescent = remove_evanescent;
  d.bandlimit = bandlimit;
  d.n_medium = n_medium;
  d.ky0 = ky0;
  d.kx0 = kx0;
  d.conj_kernel = conj_kernel;
  d.crop_y = crop_y;
  d.crop_x = crop_x;
  size_t need = 0;
  cx_status s = cx_prop2d_workspace_size(&d, &need);
  if (s == CX_OK && workspace->element_count() < need) s = CX_ERR_WORKSPACE;
  if (s == CX_OK)
    s = cx_prop2d(&d, reinterpret_cast<const cx_plane*>(planes.typed_data()), u.typed_data(), out->typed_data(),
                  nullptr, workspace->typed_data(), workspace->element_count(), stream);
  if (s != CX_OK) return ffi::Error(ffi::ErrorCode::kInternal, cx_last_error());
  return ffi::Error::Success();
}

XLA_FFI_DEFINE_HANDLER_SYMBOL(cx_prop2d_ffi, Prop2D,
                              ffi::Ffi::Bind()
                                  .Ctx<ffi::PlatformStream<cudaStream_t>>()
                                  .Arg<ffi::Buffer<ffi::C64>>()
                                  .Arg<ffi::Buffer<ffi::U8>>()
                                  .Ret<ffi::Buffer<ffi::C64>>()
                                  .Ret<ffi::Buffer<ffi::U8>>()
                                  .Attr<int32_t>("ny")
                                  .Attr<int32_t>("nx")
                                  .Attr<int32_t>("pad_y")
                                  .Attr<int32_t>("pad_x")
                                  .Attr<int32_t>("crop_y")
                                  .Attr<int32_t>("crop_x")
                                  .Attr<int32_t>("mode_same")
                                  .Attr<int32_t>("kernel")
                                  .Attr<int32_t>("precision")
                                  .Attr<int32_t>("remove_evanescent")
                                  .Attr<int32_t>("bandlimit")
                                  .Attr<int32_t>("conj_kernel")
                                  .Attr<double>("n_medium")
                                  .Attr<double>("ky0")
                                  .Attr<double>("kx0"));
