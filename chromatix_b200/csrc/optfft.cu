// C API of the chirped optical FFT (kernels in optfft.cuh).
#include "optfft.cuh"

namespace cx {

static cx_status opt_args(const cx_optfft_desc* d, OptArgs* a) {
  if (!d || d->ny <= 0 || d->nx <= 0 || d->pad_y < 0 || d->pad_x < 0 || d->crop_y < 0 || d->crop_x < 0 ||
      d->n_wv <= 0 || d->n_in_planes <= 0 || d->n_out_planes <= 0 || d->n_out_planes % d->n_wv ||
      d->n_in_planes % d->n_wv) {
    set_error("invalid optical FFT descriptor");
    return CX_ERR_INVALID;
  }
  a->ny = d->ny;
  a->nx = d->nx;
  a->pad_y = d->pad_y;
  a->pad_x = d->pad_x;
  a->py = d->ny + 2 * d->pad_y;
  a->px = d->nx + 2 * d->pad_x;
  a->crop_y = d->crop_y;
  a->crop_x = d->crop_x;
  a->oy_n = a->py - 2 * d->crop_y;
  a->ox_n = a->px - 2 * d->crop_x;
  a->W = d->n_wv;
  a->n_in_planes = d->n_in_planes;
  a->n_out_planes = d->n_out_planes;
  a->precision = d->precision;
  if (a->oy_n <= 0 || a->ox_n <= 0) {
    set_error("crop removes the whole field");
    return CX_ERR_INVALID;
  }
  if (!size_supported(a->py) || !size_supported(a->px)) {
    set_error("optical FFT grid %dx%d: FFT length not supported", a->py, a->px);
    return CX_ERR_UNSUPPORTED;
  }
  return CX_OK;
}

}  // namespace cx

using namespace cx;

extern "C" cx_status cx_optfft_workspace_size(const cx_optfft_desc* d, size_t* bytes) {
  OptArgs a;
  cx_status s = opt_args(d, &a);
  if (s != CX_OK) return s;
  if (!bytes) return CX_ERR_INVALID;
  *bytes = sizeof(float2) * (size_t)a.n_out_planes * a.py * a.px;
  return CX_OK;
}

extern "C" cx_status cx_optical_fft(const cx_optfft_desc* d, const cx_fft_plane* planes_dev, const void* u_in,
                                    void* u_out, void* workspace, size_t workspace_bytes, cx_stream_t stream) {
  OptArgs a;
  cx_status s = opt_args(d, &a);
  if (s != CX_OK) return s;
  if (!planes_dev || !u_in || !u_out || !workspace) {
    set_error("null pointer argument");
    return CX_ERR_INVALID;
  }
  const size_t need = sizeof(float2) * (size_t)a.n_out_planes * a.py * a.px;
  if (workspace_bytes < need) {
    set_error("workspace too small: %zu < %zu", workspace_bytes, need);
    return CX_ERR_WORKSPACE;
  }
  a.planes = planes_dev;
  a.H = nullptr;
  if ((s = ensure_twiddles(&a.twg)) != CX_OK) return s;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  float2* T = static_cast<float2*>(workspace);
  if ((s = opt_dispatch_rows(a.px, static_cast<const float2*>(u_in), T, a, st)) != CX_OK) return s;
  return opt_dispatch_cols(a.py, T, static_cast<float2*>(u_out), a, st);
}

extern "C" cx_status cx_optical_fft_h(const cx_optfft_desc* d, const cx_fft_plane* planes_dev, const void* H,
                                      const void* u_in, void* u_out, void* workspace, size_t workspace_bytes,
                                      cx_stream_t stream) {
  OptArgs a;
  cx_status s = opt_args(d, &a);
  if (s != CX_OK) return s;
  if (!planes_dev || !H || !u_in || !u_out || !workspace) {
    set_error("null pointer argument");
    return CX_ERR_INVALID;
  }
  const size_t need = sizeof(float2) * (size_t)a.n_out_planes * a.py * a.px;
  if (workspace_bytes < need) {
    set_error("workspace too small: %zu < %zu", workspace_bytes, need);
    return CX_ERR_WORKSPACE;
  }
  a.planes = planes_dev;
  a.H = static_cast<const float2*>(H);
  if ((s = ensure_twiddles(&a.twg)) != CX_OK) return s;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  float2* T = static_cast<float2*>(workspace);
  if ((s = opt_dispatch_rows(a.px, static_cast<const float2*>(u_in), T, a, st)) != CX_OK) return s;
  return opt_dispatch_cols(a.py, T, static_cast<float2*>(u_out), a, st);
}
