// C API of the plane-wise Fourier convolution with the sensor's plane sum
// (kernels in conv.cuh).
#include "conv.cuh"

namespace cx {

template <int M>
static cx_status launch_rows(const ConvArgs& a, cudaStream_t st) {
  using C = RowCfg<M>;
  auto k = k_conv_rows<M>;
  CX_CUDA_TRY(set_smem(k, C::SMEM));
  const long items = ((long)a.zc * 2 * a.h + C::TEAMS - 1) / C::TEAMS;
  k<<<persistent_grid(k, C::THREADS, C::SMEM, items), C::THREADS, C::SMEM, st>>>(a);
  CX_LAUNCH_CHECK();
  return CX_OK;
}

template <int P>
static cx_status launch_cols(const ConvArgs& a, cudaStream_t st) {
  using Q = ConvColCfg<P>;
  auto k = k_conv_cols<P>;
  CX_CUDA_TRY(set_smem(k, Q::SMEM));
  const long items = (a.NC + Q::V - 1) / Q::V;
  k<<<persistent_grid(k, Q::THREADS, Q::SMEM, items), Q::THREADS, Q::SMEM, st>>>(a);
  CX_LAUNCH_CHECK();
  return CX_OK;
}

template <int P>
static cx_status launch_fin_cols(const ConvArgs& a, cudaStream_t st) {
  using C = RowCfg<P>;
  auto k = k_conv_fin_cols<P>;
  CX_CUDA_TRY(set_smem(k, C::SMEM));
  const long items = ((long)a.NC + C::TEAMS - 1) / C::TEAMS;
  k<<<persistent_grid(k, C::THREADS, C::SMEM, items), C::THREADS, C::SMEM, st>>>(a);
  CX_LAUNCH_CHECK();
  return CX_OK;
}

template <int M>
static cx_status launch_fin_rows(const ConvArgs& a, cudaStream_t st) {
  using Q = ConvFinCfg<M>;
  auto k = k_conv_fin_rows<M>;
  CX_CUDA_TRY(set_smem(k, Q::SMEM));
  const long items = (a.h + Q::V - 1) / Q::V;
  k<<<persistent_grid(k, Q::THREADS, Q::SMEM, items), Q::THREADS, Q::SMEM, st>>>(a);
  CX_LAUNCH_CHECK();
  return CX_OK;
}

#define CX_CONV_DISPATCH_(NAME, FN, VAR)                 \
  cx_status NAME(int VAR, const ConvArgs& a, cudaStream_t st) { \
    switch (VAR) {                                       \
      CX_CONV_SIZES(CX_CONV_CASE_)                       \
    }                                                    \
    set_error("convolution length %d is not supported", VAR); \
    return CX_ERR_UNSUPPORTED;                           \
  }

#define CX_CONV_CASE_(N) \
  case N:                \
    return launch_rows<N>(a, st);
CX_CONV_DISPATCH_(conv_dispatch_rows, launch_rows, m)
#undef CX_CONV_CASE_
#define CX_CONV_CASE_(N) \
  case N:                \
    return launch_cols<N>(a, st);
CX_CONV_DISPATCH_(conv_dispatch_cols, launch_cols, p)
#undef CX_CONV_CASE_
#define CX_CONV_CASE_(N) \
  case N:                \
    return launch_fin_cols<N>(a, st);
CX_CONV_DISPATCH_(conv_dispatch_fin_cols, launch_fin_cols, p)
#undef CX_CONV_CASE_
#define CX_CONV_CASE_(N) \
  case N:                \
    return launch_fin_rows<N>(a, st);
CX_CONV_DISPATCH_(conv_dispatch_fin_rows, launch_fin_rows, m)
#undef CX_CONV_CASE_

static int next_pow2(long v) {
  long p = 1;
  while (p < v) p <<= 1;
  return (int)p;
}

// row-spectrum chunk budget (planes of both stacks per chunk)
static constexpr size_t kConvChunkBytes = (size_t)256 << 20;

static cx_status conv_plan(const cx_conv_desc* d, ConvArgs* a, int* zc, size_t* t_bytes, size_t* total) {
  if (!d || d->n_planes <= 0 || d->h < 1 || d->w < 2) {
    set_error("invalid convolution descriptor (n_planes >= 1, h >= 1, w >= 2)");
    return CX_ERR_INVALID;
  }
  a->h = d->h;
  a->w = d->w;
  a->P = next_pow2(2L * d->h);
  a->Q = next_pow2(2L * d->w);
  a->M = a->Q / 2;
  a->NC = a->M + 1;
  if (a->P < 2 || a->P > 4096 || a->Q > 4096) {
    set_error("convolution of %dx%d needs transforms of %dx%d; at most 4096 per axis", d->h, d->w, a->P, a->Q);
    return CX_ERR_UNSUPPORTED;
  }
  a->c0y = (d->h - 1) / 2;
  a->c0x = (d->w - 1) / 2;
  a->scale = (float)(2.0 / ((double)a->P * (double)a->Q));
  const size_t plane_t = sizeof(float2) * 2 * (size_t)d->h * a->NC;
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

extern "C" cx_status cx_conv2d_same(const cx_conv_desc* d, const float* sample, const float* psf, float* out,
                                    void* workspace, size_t workspace_bytes, cx_stream_t stream) {
  ConvArgs a;
  int zc = 0;
  size_t tb = 0, total = 0;
  cx_status s = conv_plan(d, &a, &zc, &tb, &total);
  if (s != CX_OK) return s;
  if (!sample || !psf || !out || !workspace) {
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
  a.b = psf;
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
