// Device twiddle tables: exp(-2 pi i m / N) for every compiled length N,
// followed by the w^(4m) copy used by the radix-8/16 stages (tw_len(N)
// entries per length), computed on the host in FP64 and rounded to float.
#include <cmath>
#include <mutex>
#include <vector>

#include "host.cuh"

namespace cx {

static __device__ float2 g_twiddles[kTwTotal];

cx_status ensure_twiddles(const float2** table) {
  static std::mutex mu;
  static const float2* addr[64] = {nullptr};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    set_error("no current CUDA device");
    return CX_ERR_CUDA;
  }
  std::lock_guard<std::mutex> lock(mu);
  if (addr[dev]) {
    if (table) *table = addr[dev];
    return CX_OK;
  }
  static std::vector<float2> host;
  if (host.empty()) {
    host.resize(kTwTotal);
    const double pi = 3.141592653589793238462643383279502884;
    for (int i = 0; i < kNumSizes; ++i) {
      const int N = kSizes[i];
      float2* t = host.data() + tw_offset(N);
      for (int m = 0; m < tw_len(N); ++m) {
        const long e = m < N ? m : (4L * (m - N)) % N;
        // exact symmetric reduction keeps the argument small: angle = 2 pi e / N
        const double a = 2.0 * pi * (double)e / (double)N;
        t[m] = make_float2((float)std::cos(a), (float)(-std::sin(a)));
      }
    }
  }
  // synchronous copy: visible to every stream once this returns; a first call
  // inside a stream capture is refused by the runtime (call cx_init first)
  CX_CUDA_TRY(cudaMemcpyToSymbol(g_twiddles, host.data(), sizeof(float2) * kTwTotal));
  void* p = nullptr;
  CX_CUDA_TRY(cudaGetSymbolAddress(&p, g_twiddles));
  addr[dev] = static_cast<const float2*>(p);
  if (table) *table = addr[dev];
  return CX_OK;
}

}  // namespace cx

extern "C" cx_status cx_init(void) { return cx::ensure_twiddles(nullptr); }
