// C API of the modified-Born-series iteration (kernels in mbs.cuh).
#include <cmath>

#include "mbs.cuh"

namespace cx {

bool mbs_size_supported(int n);

static cx_status mbs_args(const cx_mbs_desc* d, MbsArgs* a) {
  if (!d || d->X <= 0 || d->Y <= 0 || d->Z <= 0 || !(d->spacing > 0.0) || !(d->k0 > 0.0)) {
    set_error("invalid MBS descriptor");
    return CX_ERR_INVALID;
  }
  if (!mbs_size_supported(d->X) || !mbs_size_supported(d->Y) || !mbs_size_supported(d->Z)) {
    set_error("MBS grid %dx%dx%d: length not supported", d->X, d->Y, d->Z);
    return CX_ERR_UNSUPPORTED;
  }
  a->X = d->X;
  a->Y = d->Y;
  a->Z = d->Z;
  a->vox = (long)d->X * d->Y * d->Z;
  a->s = make_float2((float)d->s_re, (float)d->s_im);
  a->kb2 = make_float2((float)d->kb2_re, (float)d->kb2_im);
  const double twopi = 6.283185307179586476925286766559;
  // k' = 2 pi fftfreq(N) / (spacing k0) = (2 pi / (N spacing k0)) * freq index
  a->kfx = (float)(twopi / (d->X * d->spacing * d->k0));
  a->kfy = (float)(twopi / (d->Y * d->spacing * d->k0));
  a->kfz = (float)(twopi / (d->Z * d->spacing * d->k0));
  return ensure_twiddles(&a->twg);
}

// G applied to buf (after the z pass has filled it): FFT_y, X pass, IFFT_y
static cx_status mbs_middle(const MbsArgs& a, cudaStream_t st) {
  cx_status s;
  // y: per (component, ix) plane (Y rows of Z), element stride Z, inner Z
  if ((s = mbs_dispatch_cols(a.Y, false, a, 3L * a.X, a.Z, (long)a.Y * a.Z, a.Z, st)) != CX_OK) return s;
  if ((s = mbs_dispatch_x(a.X, a, st)) != CX_OK) return s;
  return mbs_dispatch_cols(a.Y, true, a, 3L * a.X, a.Z, (long)a.Y * a.Z, a.Z, st);
}

}  // namespace cx

using namespace cx;

extern "C" cx_status cx_mbs_workspace_size(const cx_mbs_desc* d, size_t* bytes) {
  MbsArgs a{};  // pointers a call does not set stay null
  cx_status s = mbs_args(d, &a);
  if (s != CX_OK && s != CX_ERR_CUDA) return s;
  if (!bytes) return CX_ERR_INVALID;
  *bytes = sizeof(float2) * 3 * (size_t)a.vox;
  return CX_OK;
}

extern "C" cx_status cx_mbs_precondition(const cx_mbs_desc* d, const void* eps, const void* src, void* prec_y,
                                         void* workspace, size_t workspace_bytes, cx_stream_t stream) {
  MbsArgs a{};  // pointers a call does not set stay null
  cx_status s = mbs_args(d, &a);
  if (s != CX_OK) return s;
  if (!eps || !src || !prec_y || !workspace || workspace_bytes < sizeof(float2) * 3 * (size_t)a.vox) {
    set_error("invalid MBS precondition arguments");
    return CX_ERR_INVALID;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  a.eps = static_cast<const float2*>(eps);
  a.x = static_cast<const float2*>(src);
  a.buf = static_cast<float2*>(workspace);
  a.x_new = static_cast<float2*>(prec_y);
  if ((s = mbs_dispatch_z(a.Z, MBS_Z_SCALE, a, st)) != CX_OK) return s;
  if ((s = mbs_middle(a, st)) != CX_OK) return s;
  return mbs_dispatch_z(a.Z, MBS_ZI_PREC, a, st);
}

extern "C" cx_status cx_mbs_iterate(const cx_mbs_desc* d, const void* eps, const void* prec_y, const void* x,
                                    void* x_new, double* acc, void* workspace, size_t workspace_bytes,
                                    cx_stream_t stream) {
  MbsArgs a{};  // pointers a call does not set stay null
  cx_status s = mbs_args(d, &a);
  if (s != CX_OK) return s;
  if (!eps || !prec_y || !x || !x_new || !acc || !workspace ||
      workspace_bytes < sizeof(float2) * 3 * (size_t)a.vox || x == x_new) {
    set_error("invalid MBS iterate arguments (x and x_new must differ)");
    return CX_ERR_INVALID;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  a.eps = static_cast<const float2*>(eps);
  a.x = static_cast<const float2*>(x);
  a.prec_y = static_cast<const float2*>(prec_y);
  a.buf = static_cast<float2*>(workspace);
  a.x_new = static_cast<float2*>(x_new);
  a.acc = acc;
  CX_CUDA_TRY(cudaMemsetAsync(acc, 0, 2 * sizeof(double), st));
  if ((s = mbs_dispatch_z(a.Z, MBS_Z_DISC, a, st)) != CX_OK) return s;
  if ((s = mbs_middle(a, st)) != CX_OK) return s;
  return mbs_dispatch_z(a.Z, MBS_ZI_STEP, a, st);
}

extern "C" cx_status cx_mbs_forward(const cx_mbs_desc* d, const void* eps, const void* x, void* out, void* workspace,
                                    size_t workspace_bytes, cx_stream_t stream) {
  MbsArgs a{};  // pointers a call does not set stay null
  cx_status s = mbs_args(d, &a);
  if (s != CX_OK) return s;
  if (!eps || !x || !out || !workspace || workspace_bytes < sizeof(float2) * 3 * (size_t)a.vox || x == out) {
    set_error("invalid MBS forward arguments (x and out must differ)");
    return CX_ERR_INVALID;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  a.eps = static_cast<const float2*>(eps);
  a.x = static_cast<const float2*>(x);
  a.prec_y = static_cast<const float2*>(x);  // unused when forward_only
  a.buf = static_cast<float2*>(workspace);
  a.x_new = static_cast<float2*>(out);
  a.acc = nullptr;
  a.forward_only = 1;
  if ((s = mbs_dispatch_z(a.Z, MBS_Z_DISC, a, st)) != CX_OK) return s;
  if ((s = mbs_middle(a, st)) != CX_OK) return s;
  return mbs_dispatch_z(a.Z, MBS_ZI_STEP, a, st);
}
