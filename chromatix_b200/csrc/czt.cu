// C API of the chirp-Z transform (kernels in czt.cuh).
#include <cmath>
#include <mutex>

#include "czt.cuh"

namespace cx {

// chirp filter c[i] = w^(-(i - n + 1)^2 / 2) / L for i < n + m - 1, 0 beyond
// (utils/czt.py:38-40), FP64 sin/cos: it is evaluated once per call
__global__ void k_czt_filter(float2* __restrict__ c, int n, int m, int L, double tw, double lw) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < L; i += gridDim.x * blockDim.x) {
    float2 v = make_float2(0.f, 0.f);
    if (i < n + m - 1) {
      const double d = (double)(i - (n - 1));
      const double ph = -tw * 0.5 * d * d;
      const double mag = exp(-lw * 0.5 * d * d) / (double)L;
      double sd, cd;
      sincos(ph, &sd, &cd);
      v = make_float2((float)(mag * cd), (float)(mag * sd));
    }
    c[i] = v;
  }
}

static int czt_length(int n, int m, int L) {
  if (L > 0) return L;
  const int need = n + m - 1;
  for (int i = 0; i < kNumSizes; ++i)
    if (kSizes[i] >= need) return kSizes[i];
  return -1;
}

static cx_status czt_args(const cx_czt_desc* d, CztArgs* a) {
  if (!d || d->n <= 0 || d->m <= 0 || d->n_vec <= 0 || d->inner <= 0 || d->n_vec % d->inner) {
    set_error("invalid CZT descriptor");
    return CX_ERR_INVALID;
  }
  const int L = czt_length(d->n, d->m, d->L);
  if (L < d->n + d->m - 1 || !size_supported_1d(L)) {
    set_error("CZT needs an FFT length >= n + m - 1 = %d (largest compiled length 8192)", d->n + d->m - 1);
    return CX_ERR_UNSUPPORTED;
  }
  if (d->layout == 1 && (d->in_istride != 1 || d->out_istride != 1)) {
    set_error("column-tile CZT needs unit inner strides");
    return CX_ERR_INVALID;
  }
  a->n = d->n;
  a->m = d->m;
  a->L = L;
  a->n_vec = d->n_vec;
  a->inner = d->inner;
  a->in_ostride = d->in_ostride;
  a->in_istride = d->in_istride;
  a->in_estride = d->in_estride;
  a->out_ostride = d->out_ostride;
  a->out_istride = d->out_istride;
  a->out_estride = d->out_estride;
  a->ta = std::atan2(d->a_im, d->a_re);
  a->tw = std::atan2(d->w_im, d->w_re);
  a->la = std::log(std::hypot(d->a_re, d->a_im));
  a->lw = std::log(std::hypot(d->w_re, d->w_im));
  a->modN = d->mod_n;
  a->scale = d->scale;
  if (d->adjoint) {
    // x'[j] = sum_k conj(scale M_k a^-j w^jk) y'[k], M_k = w^(-N k) a^N (or 1):
    // a Bluestein transform of m inputs onto n outputs with w' = conj(w),
    // input factor conj(M_k) conj(w)^(k^2/2) (a' = conj(w)^N), output factor
    // conj(w)^(j^2/2) conj(a)^(-j) [conj(a)^N] scale
    const double ta = a->ta, la = a->la, tw = a->tw, lw = a->lw;
    const double N = d->mod_n >= 0 ? (double)d->mod_n : 0.0;
    a->n = d->m;
    a->m = d->n;
    a->tw = -tw;
    a->lw = lw;
    a->ta = -N * tw;
    a->la = N * lw;
    a->modN = -1;
    a->gb_l = -la;
    a->gb_t = ta;
    a->c_l = N * la;
    a->c_t = -N * ta;
  }
  return CX_OK;
}

}  // namespace cx

using namespace cx;

extern "C" cx_status cx_czt_workspace_size(const cx_czt_desc* d, size_t* bytes) {
  CztArgs a;
  cx_status s = czt_args(d, &a);
  if (s != CX_OK) return s;
  if (!bytes) return CX_ERR_INVALID;
  *bytes = 2 * sizeof(float2) * (size_t)a.L;
  return CX_OK;
}

extern "C" cx_status cx_czt(const cx_czt_desc* d, const void* x, void* y, void* workspace, size_t workspace_bytes,
                            cx_stream_t stream) {
  CztArgs a;
  cx_status s = czt_args(d, &a);
  if (s != CX_OK) return s;
  if (!x || !y || !workspace) {
    set_error("null pointer argument");
    return CX_ERR_INVALID;
  }
  if (workspace_bytes < 2 * sizeof(float2) * (size_t)a.L) {
    set_error("workspace too small");
    return CX_ERR_WORKSPACE;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if ((s = ensure_twiddles(&a.twg)) != CX_OK) return s;
  float2* c = static_cast<float2*>(workspace);
  float2* chat = c + a.L;
  k_czt_filter<<<(a.L + 255) / 256, 256, 0, st>>>(c, a.n, a.m, a.L, a.tw, a.lw);
  CX_LAUNCH_CHECK();
  if ((s = cx_fft1d(c, chat, a.L, 1, 0, stream)) != CX_OK) return s;
  a.chat = chat;
  a.x = static_cast<const float2*>(x);
  a.y = static_cast<float2*>(y);
  return d->layout == 1 ? czt_dispatch_cols(a.L, a, st) : czt_dispatch_rows(a.L, a, st);
}

// ---------------------------------------------------------------------------
// cx_czt_noalloc: the same transform with its scratch in a static device buffer
// ---------------------------------------------------------------------------

namespace cx {

// chirp filter (L entries) followed by its spectrum (L entries); 64 KiB.
// Every entry a call reads is written earlier in the same call (the filter
// kernel writes zeros past n + m - 1), so nothing has to start at zero.
constexpr int kCztNoAllocMaxL = 4096;
static __device__ __align__(256) float2 g_czt_scratch[2 * kCztNoAllocMaxL];

// Address of g_czt_scratch on the current device, looked up once per device.
static cx_status czt_noalloc_scratch(float2** out) {
  static std::mutex mu;
  static float2* addr[64] = {nullptr};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    set_error("cx_czt_noalloc: no current CUDA device");
    return CX_ERR_CUDA;
  }
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress((void**)&p, g_czt_scratch);
    if (e != cudaSuccess || !p) {
      set_error("cx_czt_noalloc: cudaGetSymbolAddress of the static scratch failed: %s", cudaGetErrorString(e));
      return CX_ERR_CUDA;
    }
    addr[dev] = static_cast<float2*>(p);
  }
  *out = addr[dev];
  return CX_OK;
}

}  // namespace cx

extern "C" cx_status cx_czt_noalloc(const cx_czt_desc* d, const void* x, void* y, cx_stream_t stream) {
  if (d && (d->L > kCztNoAllocMaxL || (int64_t)d->n + d->m - 1 > kCztNoAllocMaxL)) {
    set_error("cx_czt_noalloc: FFT length %d (n + m - 1 = %lld) exceeds the static scratch, which holds L <= %d",
              d->L, (long long)d->n + d->m - 1, kCztNoAllocMaxL);
    return CX_ERR_UNSUPPORTED;
  }
  CztArgs a;
  cx_status s = czt_args(d, &a);
  if (s != CX_OK) return s;
  if (a.L > kCztNoAllocMaxL) {
    set_error("cx_czt_noalloc: FFT length %d exceeds the static scratch, which holds L <= %d", a.L, kCztNoAllocMaxL);
    return CX_ERR_UNSUPPORTED;
  }
  if (!x || !y) {
    set_error("null pointer argument");
    return CX_ERR_INVALID;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if ((s = ensure_twiddles(&a.twg)) != CX_OK) return s;
  float2* c = nullptr;
  if ((s = czt_noalloc_scratch(&c)) != CX_OK) return s;
  float2* chat = c + a.L;
  k_czt_filter<<<(a.L + 255) / 256, 256, 0, st>>>(c, a.n, a.m, a.L, a.tw, a.lw);
  CX_LAUNCH_CHECK();
  if ((s = cx_fft1d(c, chat, a.L, 1, 0, stream)) != CX_OK) return s;
  a.chat = chat;
  a.x = static_cast<const float2*>(x);
  a.y = static_cast<float2*>(y);
  return d->layout == 1 ? czt_dispatch_cols(a.L, a, st) : czt_dispatch_rows(a.L, a, st);
}
