// C ABI plumbing: error strings, device info, batched 1D FFT, intensity.
#include <map>
#include <mutex>
#include <utility>

#include "host.cuh"

namespace cx {

static thread_local char g_err[512] = "";

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

KernelFacts& kernel_facts_slot(const void* kernel, int device) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, KernelFacts> reg;  // node-based: references stay valid
  std::lock_guard<std::mutex> lock(mu);
  return reg[std::make_pair(kernel, device)];
}

int sm_count() {
  static int cache[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (cache[dev] == 0) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    cache[dev] = n;
  }
  return cache[dev];
}

// ---------------------------------------------------------------------------
// batched 1D FFT along contiguous rows (engine test / utility)
// ---------------------------------------------------------------------------
template <int N, bool INV>
__global__ void __launch_bounds__(RowCfg<N>::THREADS, RowCfg<N>::MINB) k_fft1d(const float2* __restrict__ in, float2* __restrict__ out,
                                                             long batch, const float2* __restrict__ twg) {
  using C = RowCfg<N>;
  extern __shared__ float2 sm[];
  float2* tw = sm;
  load_twiddles<N>(tw, twg, threadIdx.x, blockDim.x);
  __syncthreads();
  const int team = threadIdx.x / C::LPV, lane = threadIdx.x % C::LPV;
  float2* s = sm + C::TW + team * Plan<N>::LEN;
  const float scale = INV ? 1.0f / (float)N : 1.0f;
  for (long base = (long)blockIdx.x * C::TEAMS; base < batch; base += (long)gridDim.x * C::TEAMS) {
    const long item = base + team;
    const bool valid = item < batch;
    const float2* src = in + (size_t)item * N;
    float2* dst = out + (size_t)item * N;
    auto load = [&](int n) -> float2 { return valid ? src[n] : make_float2(0.f, 0.f); };
    auto store = [&](int k, float2 v, int) {
      if (valid) dst[k] = cscale(v, scale);
    };
    team_fft<N, INV>(s, tw, lane, team, load, store);
  }
}

template <int N>
static cx_status launch_fft1d(const float2* in, float2* out, long batch, bool inv, const float2* twg,
                              cudaStream_t st) {
  using C = RowCfg<N>;
  const long items = (batch + C::TEAMS - 1) / C::TEAMS;
  if (inv) {
    auto k = k_fft1d<N, true>;
    CX_CUDA_TRY(set_smem(k, C::SMEM));
    k<<<persistent_grid(k, C::THREADS, C::SMEM, items), C::THREADS, C::SMEM, st>>>(in, out, batch, twg);
  } else {
    auto k = k_fft1d<N, false>;
    CX_CUDA_TRY(set_smem(k, C::SMEM));
    k<<<persistent_grid(k, C::THREADS, C::SMEM, items), C::THREADS, C::SMEM, st>>>(in, out, batch, twg);
  }
  CX_LAUNCH_CHECK();
  return CX_OK;
}

// ---------------------------------------------------------------------------
// intensity readout
// ---------------------------------------------------------------------------
__global__ void k_intensity(const float2* __restrict__ u, long n_pix, int W, const double* __restrict__ dens,
                            float* __restrict__ out) {
  float d[8];
  for (int w = 0; w < W && w < 8; ++w) d[w] = (float)dens[w];
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n_pix; i += (long)gridDim.x * blockDim.x) {
    float acc = 0.f;
    if (W == 1) {
      acc = cabs2(u[i]) * d[0];
    } else {
      for (int w = 0; w < W; ++w) acc += d[w] * cabs2(u[(size_t)i * W + w]);
    }
    out[i] = acc;
  }
}

}  // namespace cx

using namespace cx;

extern "C" const char* cx_last_error(void) { return g_err; }

extern "C" int32_t cx_version(void) { return 100; }

extern "C" int32_t cx_fft_size_supported(int32_t n) { return size_supported(n) ? 1 : 0; }

extern "C" cx_status cx_fft1d(const void* in, void* out, int32_t n, int64_t batch, int32_t inverse,
                              cx_stream_t stream) {
  if (!in || !out || batch < 0) {
    set_error("invalid fft1d arguments");
    return CX_ERR_INVALID;
  }
  if (batch == 0) return CX_OK;
  const float2* twg = nullptr;
  cx_status s = ensure_twiddles(&twg);
  if (s != CX_OK) return s;
  const float2* i = static_cast<const float2*>(in);
  float2* o = static_cast<float2*>(out);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  switch (n) {
#define CX_CASE_(N) \
  case N:           \
    return launch_fft1d<N>(i, o, batch, inverse != 0, twg, st);
    CX_FOR_EACH_1D_SIZE(CX_CASE_)
#undef CX_CASE_
  }
  set_error("FFT length %d is not supported", n);
  return CX_ERR_UNSUPPORTED;
}

extern "C" cx_status cx_intensity(const void* u, int64_t n_pix, int32_t n_wv, const double* density_dev, float* out,
                                  cx_stream_t stream) {
  if (!u || !out || !density_dev || n_pix < 0 || n_wv < 1 || n_wv > 8) {
    set_error("invalid intensity arguments (1 <= n_wv <= 8)");
    return CX_ERR_INVALID;
  }
  if (n_pix == 0) return CX_OK;
  int grid = (int)((n_pix + 255) / 256);
  if (grid > sm_count() * 8) grid = sm_count() * 8;
  k_intensity<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(static_cast<const float2*>(u), n_pix, n_wv,
                                                                      density_dev, out);
  CX_LAUNCH_CHECK();
  return CX_OK;
}
