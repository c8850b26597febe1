// C API of the Fourier-multiplier propagation (kernels in prop2d.cuh).
#include "prop2d.cuh"

namespace cx {

// --------------------------------------------------------------------------
// propagator materialisation (compute_*_propagator)
// --------------------------------------------------------------------------
__global__ void k_fill_propagator(float2* __restrict__ H, Prop2DArgs a) {
  const long per = (long)a.py * a.px;
  const long total = per * a.n_out_planes;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int q = (int)(i / per);
    const int ky = (int)((i % per) / a.px), kx = (int)(i % a.px);
    H[i] = prop_kernel(ky, kx, a, a.planes[q]);
  }
}


static cx_status make_args(const cx_prop2d_desc* d, Prop2DArgs* a) {
  if (!d) {
    set_error("null descriptor");
    return CX_ERR_INVALID;
  }
  if (d->ny <= 0 || d->nx <= 0 || d->pad_y < 0 || d->pad_x < 0 || d->n_wv <= 0 || d->n_in_planes <= 0 ||
      d->n_out_planes <= 0 || d->n_in_planes % d->n_wv || d->n_out_planes % d->n_wv) {
    set_error("invalid propagation shape (ny=%d nx=%d pad=%d,%d wv=%d in=%d out=%d)", d->ny, d->nx, d->pad_y,
              d->pad_x, d->n_wv, d->n_in_planes, d->n_out_planes);
    return CX_ERR_INVALID;
  }
  if (d->kernel < 0 || d->kernel > 3 || d->precision < 0 || d->precision > 2) {
    set_error("invalid kernel kind or precision");
    return CX_ERR_INVALID;
  }
  if (d->precision == CX_PREC_SPLIT16 &&
      !prop_tc_supported(d->ny + 2 * d->pad_y, d->nx + 2 * d->pad_x)) {
    set_error("CX_PREC_SPLIT16 propagation: padded grid %dx%d not compiled in (1024 or 1280 rows, columns a "
              "multiple of 8)", d->ny + 2 * d->pad_y, d->nx + 2 * d->pad_x);
    return CX_ERR_UNSUPPORTED;
  }
  a->ny = d->ny;
  a->nx = d->nx;
  a->pad_y = d->pad_y;
  a->pad_x = d->pad_x;
  a->py = d->ny + 2 * d->pad_y;
  a->px = d->nx + 2 * d->pad_x;
  a->W = d->n_wv;
  a->n_in_planes = d->n_in_planes;
  a->n_out_planes = d->n_out_planes;
  if (d->crop_y < 0 || d->crop_x < 0 || 2 * d->crop_y >= a->py || 2 * d->crop_x >= a->px ||
      (d->mode_same && (d->crop_y || d->crop_x))) {
    set_error("invalid crop (%d, %d) of the padded grid %dx%d (crop applies to mode_same = 0 only)", d->crop_y,
              d->crop_x, a->py, a->px);
    return CX_ERR_INVALID;
  }
  if (d->mode_same) {
    a->out_y0 = d->pad_y;
    a->out_ny = d->ny;
    a->out_x0 = d->pad_x;
    a->out_nx = d->nx;
  } else {
    a->out_y0 = d->crop_y;
    a->out_ny = a->py - 2 * d->crop_y;
    a->out_x0 = d->crop_x;
    a->out_nx = a->px - 2 * d->crop_x;
  }
  a->kernel = d->kernel;
  a->precision = d->precision;
  a->remove_evanescent = d->remove_evanescent;
  a->bandlimit = d->bandlimit;
  a->n_med = d->n_medium;
  a->ky0 = d->ky0;
  a->kx0 = d->kx0;
  a->na_f2 = -1.0;
  a->precise = 0;
  a->conj_h = d->conj_kernel ? 1 : 0;
  a->twg = nullptr;
  a->planes = nullptr;
  a->H = nullptr;
  if (!size_supported_prop(a->py) || !size_supported_prop(a->px)) {
    set_error("padded grid %dx%d: FFT length not supported", a->py, a->px);
    return CX_ERR_UNSUPPORTED;
  }
  return CX_OK;
}

static size_t ws_T_bytes(const Prop2DArgs& a) { return sizeof(float2) * (size_t)a.n_in_planes * a.ny * a.px; }
static size_t ws_T2_bytes(const Prop2DArgs& a) { return sizeof(float2) * (size_t)a.n_out_planes * a.out_ny * a.px; }
static size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

}  // namespace cx

using namespace cx;

extern "C" cx_status cx_prop2d_workspace_size(const cx_prop2d_desc* d, size_t* bytes) {
  Prop2DArgs a;
  cx_status s = make_args(d, &a);
  if (s != CX_OK) return s;
  if (!bytes) {
    set_error("null bytes pointer");
    return CX_ERR_INVALID;
  }
  *bytes = align256(ws_T_bytes(a)) + align256(ws_T2_bytes(a));
  return CX_OK;
}

extern "C" cx_status cx_prop2d(const cx_prop2d_desc* d, const cx_plane* planes_dev, const void* u_in, void* u_out,
                               const void* H, void* workspace, size_t workspace_bytes, cx_stream_t stream) {
  Prop2DArgs a;
  cx_status s = make_args(d, &a);
  if (s != CX_OK) return s;
  if (!planes_dev || !u_in || !u_out || !workspace) {
    set_error("null pointer argument");
    return CX_ERR_INVALID;
  }
  if (d->kernel == CX_KERNEL_EXPLICIT && !H) {
    set_error("explicit propagator requested but H is null");
    return CX_ERR_INVALID;
  }
  const size_t need = align256(ws_T_bytes(a)) + align256(ws_T2_bytes(a));
  if (workspace_bytes < need) {
    set_error("workspace too small: %zu < %zu", workspace_bytes, need);
    return CX_ERR_WORKSPACE;
  }
  a.planes = planes_dev;
  a.H = static_cast<const float2*>(H);
  if ((s = ensure_twiddles(&a.twg)) != CX_OK) return s;
  float2* T = static_cast<float2*>(workspace);
  float2* T2 = reinterpret_cast<float2*>(static_cast<char*>(workspace) + align256(ws_T_bytes(a)));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if ((s = prop_rows_fwd(static_cast<const float2*>(u_in), T, a, st)) != CX_OK) return s;
  if ((s = prop_cols(a.py, T, T2, a, st)) != CX_OK) return s;
  return prop_rows_inv(T2, static_cast<float2*>(u_out), a, st);
}

extern "C" cx_status cx_prop2d_ptrs(const cx_prop2d_desc* d, const cx_plane* planes_dev,
                                    const void* const* u_in_ptrs_dev, void* const* u_out_ptrs_dev, const void* H,
                                    void* workspace, size_t workspace_bytes, cx_stream_t stream) {
  Prop2DArgs a;
  cx_status s = make_args(d, &a);
  if (s != CX_OK) return s;
  if (!planes_dev || !u_in_ptrs_dev || !u_out_ptrs_dev || !workspace) {
    set_error("null pointer argument");
    return CX_ERR_INVALID;
  }
  if (d->kernel == CX_KERNEL_EXPLICIT && !H) {
    set_error("explicit propagator requested but H is null");
    return CX_ERR_INVALID;
  }
  const size_t need = align256(ws_T_bytes(a)) + align256(ws_T2_bytes(a));
  if (workspace_bytes < need) {
    set_error("workspace too small: %zu < %zu", workspace_bytes, need);
    return CX_ERR_WORKSPACE;
  }
  a.planes = planes_dev;
  a.H = static_cast<const float2*>(H);
  a.in_ptrs = reinterpret_cast<const float2* const*>(u_in_ptrs_dev);
  a.out_ptrs = reinterpret_cast<float2* const*>(u_out_ptrs_dev);
  if ((s = ensure_twiddles(&a.twg)) != CX_OK) return s;
  float2* T = static_cast<float2*>(workspace);
  float2* T2 = reinterpret_cast<float2*>(static_cast<char*>(workspace) + align256(ws_T_bytes(a)));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if ((s = prop_rows_fwd(nullptr, T, a, st)) != CX_OK) return s;
  if ((s = prop_cols(a.py, T, T2, a, st)) != CX_OK) return s;
  return prop_rows_inv(T2, nullptr, a, st);
}

extern "C" cx_status cx_fill_propagator(const cx_prop2d_desc* d, const cx_plane* planes_dev, void* H_out,
                                        cx_stream_t stream) {
  Prop2DArgs a;
  cx_status s = make_args(d, &a);
  if (s != CX_OK && s != CX_ERR_UNSUPPORTED) return s;
  if (!planes_dev || !H_out || d->kernel == CX_KERNEL_EXPLICIT) {
    set_error("invalid propagator request");
    return CX_ERR_INVALID;
  }
  a.planes = planes_dev;
  const long total = (long)a.py * a.px * a.n_out_planes;
  int grid = (int)((total + 255) / 256);
  if (grid > sm_count() * 16) grid = sm_count() * 16;
  k_fill_propagator<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(static_cast<float2*>(H_out), a);
  CX_LAUNCH_CHECK();
  return CX_OK;
}
