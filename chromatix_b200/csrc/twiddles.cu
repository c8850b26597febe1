// Device twiddle tables: exp(-2 pi i m / N) for every compiled length N,
// followed by the w^(4m) copy used by the radix-8/16 stages (tw_len(N)
// entries per length), computed on the host in FP64 and rounded to float.
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include <cuda_fp16.h>

#include "host.cuh"
#include "tcgen05.cuh"

namespace cx {

static __device__ float2 g_twiddles[kTwTotal];

// DFT matrices of lengths 32 and 40 (see tc_dft_mats), 16-byte aligned
constexpr int kTcLens[] = {32, 40};
constexpr uint32_t kTcMatTotal = tc_dft_mat_bytes(32) + tc_dft_mat_bytes(40);
static __device__ uint4 g_tc_mats[kTcMatTotal / 16];
static const uint8_t* g_tc_addr[64] = {nullptr};
static __device__ int g_tc_timeouts;
static int* g_tc_timeouts_addr[64] = {nullptr};

int* tc_timeout_counter() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  return g_tc_timeouts_addr[dev];
}

// row j = output (re | im), column k = input (re | im) of the length-R DFT
// exp(-2 pi i n k / R), as tc_fft_build_b lays it out on the device
static void build_tc_mat(int R, uint8_t* dst) {
  const int K = 2 * R;
  const double pi = 3.141592653589793238462643383279502884;
  for (int j = 0; j < K; ++j)
    for (int k = 0; k < K; ++k) {
      const int n = k % R, kk = j % R, pin = k / R, pout = j / R;
      const double a = -2.0 * pi * (double)((n * kk) % R) / (double)R;
      const float v = (float)(pin == pout ? std::cos(a) : (pin == 0 ? std::sin(a) : -std::sin(a)));
      const __half h = __float2half_rn(v);
      const __half l = __float2half_rn(v - __half2float(h));
      std::memcpy(dst + tc::off_kmajor(K, j, k), &h, 2);
      std::memcpy(dst + K * K * 2 + tc::off_kmajor(K, j, k), &l, 2);
    }
}

const uint8_t* tc_dft_mats(int R) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64 || !g_tc_addr[dev]) return nullptr;
  uint32_t off = 0;
  for (int L : kTcLens) {
    if (L == R) return g_tc_addr[dev] + off;
    off += tc_dft_mat_bytes(L);
  }
  return nullptr;
}

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
  static std::vector<uint8_t> mats;
  if (mats.empty()) {
    mats.resize(kTcMatTotal);
    uint32_t off = 0;
    for (int L : kTcLens) {
      build_tc_mat(L, mats.data() + off);
      off += tc_dft_mat_bytes(L);
    }
  }
  // synchronous copies: visible to every stream once this returns; a first
  // call inside a stream capture is refused by the runtime (call cx_init first)
  CX_CUDA_TRY(cudaMemcpyToSymbol(g_twiddles, host.data(), sizeof(float2) * kTwTotal));
  CX_CUDA_TRY(cudaMemcpyToSymbol(g_tc_mats, mats.data(), kTcMatTotal));
  void* q = nullptr;
  CX_CUDA_TRY(cudaGetSymbolAddress(&q, g_tc_mats));
  g_tc_addr[dev] = static_cast<const uint8_t*>(q);
  void* c = nullptr;
  CX_CUDA_TRY(cudaGetSymbolAddress(&c, g_tc_timeouts));
  g_tc_timeouts_addr[dev] = static_cast<int*>(c);
  void* p = nullptr;
  CX_CUDA_TRY(cudaGetSymbolAddress(&p, g_twiddles));
  addr[dev] = static_cast<const float2*>(p);
  if (table) *table = addr[dev];
  return CX_OK;
}

}  // namespace cx

extern "C" cx_status cx_init(void) { return cx::ensure_twiddles(nullptr); }

extern "C" cx_status cx_tc_timeouts(int32_t* count, int32_t reset) {
  if (!count) {
    cx::set_error("null count pointer");
    return CX_ERR_INVALID;
  }
  cx_status s = cx::ensure_twiddles(nullptr);
  if (s != CX_OK) return s;
  int v = 0;
  CX_CUDA_TRY(cudaMemcpyFromSymbol(&v, cx::g_tc_timeouts, sizeof(int)));
  *count = v;
  if (reset) {
    const int zero = 0;
    CX_CUDA_TRY(cudaMemcpyToSymbol(cx::g_tc_timeouts, &zero, sizeof(int)));
  }
  return CX_OK;
}
