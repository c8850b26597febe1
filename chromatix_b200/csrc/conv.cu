// C API of the plane-wise Fourier convolution with the sensor's plane sum
// (kernels in conv.cuh).
#include "conv.cuh"

namespace cx {

#define CX_CONV_LIST_(N) N,
static constexpr int kConvP[] = {CX_CONV_P_SIZES(CX_CONV_LIST_)};
static constexpr int kConvM[] = {CX_CONV_M_SIZES(CX_CONV_LIST_)};
#undef CX_CONV_LIST_

// smallest length >= need in an ascending list (times `mul`), powers of two
// only on request; 0 if none
template <size_t K>
static int conv_len(const int (&list)[K], int mul, long need, bool pow2) {
  for (size_t i = 0; i < K; ++i) {
    const long L = (long)list[i] * mul;
    if (L >= need && (!pow2 || (L & (L - 1)) == 0)) return (int)L;
  }
  return 0;
}

// Row-spectrum chunk budget (zc planes of both stacks per chunk): large, so
// that the column pass accumulates many planes in registers per St update;
// its loads of the row spectra overlap the transforms.
static constexpr size_t kConvChunkBytes = (size_t)1 << 30;

static cx_status conv_plan(const cx_conv_desc* d, ConvArgs* a, int* zc, size_t* t_bytes, size_t* total) {
  if (!d || d->n_planes <= 0 || d->h < 1 || d->w < 1 || d->kh < 1 || d->kw < 1) {
    set_error("invalid convolution descriptor (n_planes, h, w, kh, kw >= 1)");
    return CX_ERR_INVALID;
  }
  a->h = d->h;
  a->w = d->w;
  a->kh = d->kh;
  a->kw = d->kw;
  const int H = d->h > d->kh ? d->h : d->kh;
  a->HB = H;

  const int W = d->w > d->kw ? d->w : d->kw;
  // >= h + kh - 1 (linear convolution) and >= 2 max(h, kh): the inputs then
  // fill at most the first half of every transform (first-stage zero masks)
  a->P = conv_len(kConvP, 1, 2L * H, d->pow2_lengths != 0);
  a->Q = conv_len(kConvM, 2, 2L * W, d->pow2_lengths != 0);
  if (a->P == 0 || a->Q == 0) {
    set_error("convolution of %dx%d with %dx%d needs transforms longer than 4096 per axis", d->h, d->w, d->kh,
              d->kw);
    return CX_ERR_UNSUPPORTED;
  }
  a->M = a->Q / 2;
  a->NC = a->M + 1;
  // T tiles: the column pass's width V (a power of two), at least 4 columns
  // so that a row's run in a tile fills a 32-byte sector
  const int cv = conv_col_tile(a->P);
  if (cv < 1 || (cv & (cv - 1)) != 0) {
    set_error("internal: column tile width %d for length %d", cv, a->P);
    return CX_ERR_UNSUPPORTED;
  }
  const int vt = cv > 4 ? cv : 4;
  a->vt_shift = 0;
  while ((1 << a->vt_shift) < vt) ++a->vt_shift;
  a->NT = (a->NC + vt - 1) / vt;
  a->b_plane = d->kernel_broadcast ? 0 : (long)d->kh * d->kw;
  a->c0y = (d->kh - 1) / 2;
  a->c0x = (d->kw - 1) / 2;
  a->scale = (float)(2.0 / ((double)a->P * (double)a->Q));
  const size_t plane_t = sizeof(float2) * 2 * (size_t)a->HB * a->NT * vt;
  int c = (int)(kConvChunkBytes / plane_t);
  if (c < 1) c = 1;
  if (c > d->n_planes) c = d->n_planes;
  *zc = c;
  *t_bytes = ((plane_t * c) + 255) & ~(size_t)255;
  const size_t st_bytes = ((sizeof(float2) * (size_t)a->NC * a->P) + 255) & ~(size_t)255;
  const size_t u_bytes = ((sizeof(float2) * (size_t)a->NC * d->h) + 255) & ~(size_t)255;
  *total = *t_bytes + st_bytes + u_bytes;
  return CX_OK;
}

}  // namespace cx

using namespace cx;

extern "C" cx_status cx_conv2d_workspace_size(const cx_conv_desc* d, size_t* bytes) {
  ConvArgs a;
  int zc = 0;
  size_t tb = 0, total = 0;
  cx_status s = conv_plan(d, &a, &zc, &tb, &total);
  if (s != CX_OK) return s;
  if (!bytes) return CX_ERR_INVALID;
  *bytes = total;
  return CX_OK;
}

extern "C" cx_status cx_conv2d_same(const cx_conv_desc* d, const float* sample, const float* kernel, float* out,
                                    void* workspace, size_t workspace_bytes, cx_stream_t stream) {
  ConvArgs a;
  int zc = 0;
  size_t tb = 0, total = 0;
  cx_status s = conv_plan(d, &a, &zc, &tb, &total);
  if (s != CX_OK) return s;
  if (!sample || !kernel || !out || !workspace) {
    set_error("null pointer argument");
    return CX_ERR_INVALID;
  }
  if (workspace_bytes < total) {
    set_error("workspace too small: %zu < %zu", workspace_bytes, total);
    return CX_ERR_WORKSPACE;
  }
  if ((s = ensure_twiddles(&a.twg)) != CX_OK) return s;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  char* ws = static_cast<char*>(workspace);
  a.T = reinterpret_cast<float2*>(ws);
  a.St = reinterpret_cast<float2*>(ws + tb);
  a.U = reinterpret_cast<float2*>(ws + tb + (((sizeof(float2) * (size_t)a.NC * a.P) + 255) & ~(size_t)255));
  a.a = sample;
  a.b = kernel;
  const size_t st_bytes = sizeof(float2) * (size_t)a.NC * a.P;
  const size_t img = (size_t)d->h * d->w;
  // reduce: one accumulated spectrum for all planes; otherwise one per plane
  const int groups = d->reduce ? 1 : d->n_planes;
  for (int g = 0; g < groups; ++g) {
    const int p_lo = d->reduce ? 0 : g, p_hi = d->reduce ? d->n_planes : g + 1;
    CX_CUDA_TRY(cudaMemsetAsync(a.St, 0, st_bytes, st));
    for (int z0 = p_lo; z0 < p_hi; z0 += zc) {
      a.z0 = z0;
      a.zc = (p_hi - z0) < zc ? (p_hi - z0) : zc;
      if ((s = conv_dispatch_rows(a.M, a, st)) != CX_OK) return s;
      if ((s = conv_dispatch_cols(a.P, a, st)) != CX_OK) return s;
    }
    a.out = out + (size_t)g * img;
    if ((s = conv_dispatch_fin_cols(a.P, a, st)) != CX_OK) return s;
    if ((s = conv_dispatch_fin_rows(a.M, a, st)) != CX_OK) return s;
  }
  return CX_OK;
}
