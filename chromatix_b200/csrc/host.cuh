// Host-side helpers shared by the kernel translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>

#include "../../include/cx_b200.h"
#include "fft_engine.cuh"

namespace cx {

// thread-local error message (defined in capi.cu)
void set_error(const char* fmt, ...);

#define CX_CUDA_TRY(call)                                                                  \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess) {                                                               \
      ::cx::set_error("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
      return CX_ERR_CUDA;                                                                  \
    }                                                                                      \
  } while (0)

#define CX_LAUNCH_CHECK()                                                                  \
  do {                                                                                     \
    cudaError_t e_ = cudaGetLastError();                                                   \
    if (e_ != cudaSuccess) {                                                               \
      ::cx::set_error("kernel launch failed: %s (%s:%d)", cudaGetErrorString(e_), __FILE__, __LINE__); \
      return CX_ERR_CUDA;                                                                  \
    }                                                                                      \
  } while (0)

// FFT lengths compiled into the fast path: 2^a, 3 * 2^a, 5 * 2^a, 7 * 2^a up to 4096.
#define CX_FOR_EACH_SIZE(X)                                                                          \
  X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(10) X(12) X(14) X(16) X(20) X(24) X(28) X(32) X(40) X(48)    \
  X(56) X(64) X(80) X(96) X(112) X(128) X(160) X(192) X(224) X(256) X(320) X(384) X(448) X(512)    \
  X(640) X(768) X(896) X(1024) X(1280) X(1536) X(1792) X(2048) X(2560) X(3072) X(3584) X(4096)

// Longer lengths compiled only for the 1D transform (cx_fft1d) and the
// chirp-Z passes, whose Bluestein length reaches n + m - 1 (up to 8192 for a
// 4096-point input): 2^9 3^2, 2^10 5, 2^11 3, 2^10 7, 2^13.
#define CX_FOR_EACH_LONG_SIZE(X) X(4608) X(5120) X(6144) X(7168) X(8192)
#define CX_FOR_EACH_1D_SIZE(X) CX_FOR_EACH_SIZE(X) CX_FOR_EACH_LONG_SIZE(X)
// The Fourier-multiplier propagation passes also take 8192 (a 4096^2 field
// padded by 2048 per side, the reference's high-resolution band-limited ASM
// example); a 8192-point row or column is one team of 512 lanes per CTA.
#define CX_FOR_EACH_PROP_SIZE(X) CX_FOR_EACH_SIZE(X) X(8192)

inline bool size_supported(int n) {
  switch (n) {
#define CX_CASE_(N) case N:
    CX_FOR_EACH_SIZE(CX_CASE_)
#undef CX_CASE_
    return true;
    default:
      return false;
  }
}

inline bool size_supported_prop(int n) { return size_supported(n) || n == 8192; }

inline bool size_supported_1d(int n) {
  switch (n) {
#define CX_CASE_(N) case N:
    CX_FOR_EACH_1D_SIZE(CX_CASE_)
#undef CX_CASE_
    return true;
    default:
      return false;
  }
}

// Offsets of the per-length twiddle tables inside one device array (lengths in
// CX_FOR_EACH_1D_SIZE order, tw_len(N) entries each).
#define CX_SIZE_LIST_(N) N,
constexpr int kSizes[] = {CX_FOR_EACH_1D_SIZE(CX_SIZE_LIST_)};
#undef CX_SIZE_LIST_
constexpr int kNumSizes = sizeof(kSizes) / sizeof(int);
constexpr int tw_offset(int N) {
  int off = 0;
  for (int i = 0; i < kNumSizes; ++i) {
    if (kSizes[i] == N) return off;
    off += tw_len(kSizes[i]);
  }
  return -1;
}
constexpr int tw_total() {
  int t = 0;
  for (int i = 0; i < kNumSizes; ++i) t += tw_len(kSizes[i]);
  return t;
}
constexpr int kTwTotal = tw_total();

// Device twiddle tables (twiddles.cu): ensure_twiddles() uploads them (host
// FP64 values rounded to float) once per device, synchronously, and returns
// their device address; kernels receive it in their argument structs.
cx_status ensure_twiddles(const float2** table);

// The real-expanded forward DFT matrices of the split-precision tensor-core
// transforms (lengths 32 and 40): 2R x 2R, K-major canonical layout, FP16 hi
// then lo, built on the host in FP64 and uploaded with the twiddle tables.
// Device address of length R's matrices (after ensure_twiddles), else null.
constexpr uint32_t tc_dft_mat_bytes(int R) { return 2u * (uint32_t)(2 * R) * (uint32_t)(2 * R) * 2u; }
const uint8_t* tc_dft_mats(int R);
// device counter of tensor-core MMA waits that ran out (cx_tc_timeouts)
int* tc_timeout_counter();

template <int N>
__device__ __forceinline__ void load_twiddles(float2* tw, const float2* __restrict__ table, int tid, int nthreads) {
  constexpr int off = tw_offset(N);
  static_assert(off >= 0, "length not in CX_FOR_EACH_SIZE");
  const float2* src = table + off;
  for (int m = tid; m < tw_len(N); m += nthreads) tw[m] = src[m];
}

int sm_count();  // of the current device (capi.cu)

// Register budget of the row / column kernels: about 80 registers per thread
// (min blocks per SM derived from the CTA size).
__host__ __device__ constexpr int minb_for(int threads) {
  const int b = 65536 / (threads * 80);
  return b < 1 ? 1 : b;
}

// Row kernels: about 192 threads (small CTAs: a 1024^2 pass is 1024 rows, so
// small CTAs keep all SMs busy), one team per vector, at most 15 multi-warp
// teams (named barrier ids 1..15).
template <int N>
struct RowCfg {
  static constexpr int LPV = Plan<N>::LPV;
  static constexpr int T0 = 192 / LPV > 0 ? 192 / LPV : 1;
  static constexpr int TEAMS = (LPV > 32 && T0 > 15) ? 15 : T0;
  static constexpr int THREADS = TEAMS * LPV;
  static constexpr int MINB = minb_for(THREADS);
  static constexpr int TW = tw_len(N);
  static constexpr size_t SMEM = sizeof(float2) * ((size_t)TW + (size_t)TEAMS * Plan<N>::LEN);
};

// Row kernels whose teams all run one transform per loop iteration (no
// per-team early exit): exact lane counts with CTA-wide barriers where the
// count does not tile warps, about 192 threads in whole warps.
template <int N, int TARGET = 192>
struct RowCfgX {
  static constexpr bool CTA = Plan<N>::LPV_X != Plan<N>::LPV;
  static constexpr int LPV = CTA ? Plan<N>::LPV_X : Plan<N>::LPV;
  static constexpr int T1 = TARGET / LPV > 0 ? TARGET / LPV : 1;
  static constexpr int teams_for() {
    int t = T1;
    if (CTA) {
      while ((t * LPV) % 32 != 0) ++t;
    } else if (LPV > 32 && t > 15) {
      t = 15;
    }
    return t;
  }
  static constexpr int TEAMS = teams_for();
  static constexpr int THREADS = TEAMS * LPV;
  static_assert(THREADS <= 1024, "row CTA too large");
  static constexpr int MINB = minb_for(THREADS);
  static constexpr int TW = tw_len(N);
  static constexpr size_t SMEM = sizeof(float2) * ((size_t)TW + (size_t)TEAMS * Plan<N>::LEN);
};

// Column stride (float2) of a V-column tile: a warp transposing a tile
// touches V columns x (32/V) rows, so the stride must put those 32 elements
// in distinct bank pairs: stride = 16/V (mod 16) for V <= 16, odd above.
__host__ __device__ constexpr int col_len(int N, int V) {
  int l = pad_idx(N - 1) + 1;
  if (V >= 16 || V == 1) return (l % 2 == 0) ? l + 1 : l;
  const int want = 16 / V;
  while (l % 16 != want) ++l;
  return l;
}

// Column-tile kernels: V adjacent columns per CTA, one team per column.  All
// teams of a CTA run the same transform in lockstep, so the teams can have
// the exact lane count N / R_max (no idle lanes) and synchronise with CTA-wide
// barriers (CTA = true) whenever that count does not tile warps.
template <int N, bool EXACT = true>
struct ColCfg {
  static constexpr bool CTA = EXACT && Plan<N>::LPV_X != Plan<N>::LPV;
  static constexpr int LPV = CTA ? Plan<N>::LPV_X : Plan<N>::LPV;
  // multi-warp teams: up to 4 columns, at most 1024 threads per CTA
  static constexpr int VT = 1024 / LPV >= 4 ? 4 : (1024 / LPV >= 2 ? 2 : 1);
  static constexpr int V0 = LPV < 32 ? (pow2_floor(256 / LPV) > 16 ? pow2_floor(256 / LPV) : 16) : VT;
  static constexpr int TW = tw_len(N);
  static constexpr size_t smem_for(int v) { return sizeof(float2) * ((size_t)TW + (size_t)v * col_len(N, v)); }
  static constexpr int V = smem_for(V0) <= 200 * 1024 ? V0 : (smem_for(V0 / 2) <= 200 * 1024 ? V0 / 2 : V0 / 4);
  static_assert(V >= 1 && V * LPV <= 1024, "column tile does not fit one CTA");
  static_assert(!CTA || (V * LPV) % 32 == 0, "exact-size teams must fill whole warps");
  static constexpr int LEN = col_len(N, V);
  static constexpr int THREADS = V * LPV;
  static constexpr int MINB = minb_for(THREADS);
  static constexpr size_t SMEM = smem_for(V);
};

// Copy rows [r0, r1) x columns [x0, x0 + V) of a row-major complex matrix
// (leading dimension ld) into a column tile: tile[c * LEN + pad_idx(dst(r))].
// Each thread issues four independent loads (two columns per 16-byte load
// when the row segments are 16-byte aligned) before storing them, so the
// copy is not serialised on global-memory latency.
template <int V, int LEN, class DstRow>
__device__ __forceinline__ void load_col_tile(float2* tile, const float2* __restrict__ src, size_t ld, int x0,
                                              int ncols, int r0, int r1, DstRow dst) {
  const int nr = r1 - r0;
  if (nr <= 0) return;
  const bool vec = (V % 2 == 0) && (ld % 2 == 0) && (x0 % 2 == 0);
  if (vec) {
    constexpr int PR = V / 2 > 0 ? V / 2 : 1;  // (vec is false for odd V)
    const int total = nr * PR;
    for (int base = threadIdx.x; base < total; base += 4 * blockDim.x) {
      float4 v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int idx = base + u * blockDim.x;
        const int i = idx / PR, c = (idx % PR) * 2;
        v[u] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (idx < total && x0 + c + 1 < ncols + 1) {
          if (x0 + c + 1 < ncols)
            v[u] = *reinterpret_cast<const float4*>(src + (size_t)(r0 + i) * ld + x0 + c);
          else if (x0 + c < ncols) {
            const float2 t = src[(size_t)(r0 + i) * ld + x0 + c];
            v[u] = make_float4(t.x, t.y, 0.f, 0.f);
          }
        }
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int idx = base + u * blockDim.x;
        if (idx < total) {
          const int i = idx / PR, c = (idx % PR) * 2;
          const int d = pad_idx(dst(r0 + i));
          tile[c * LEN + d] = make_float2(v[u].x, v[u].y);
          tile[(c + 1) * LEN + d] = make_float2(v[u].z, v[u].w);
        }
      }
    }
  } else {
    const int total = nr * V;
    for (int base = threadIdx.x; base < total; base += 4 * blockDim.x) {
      float2 v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int idx = base + u * blockDim.x;
        const int i = idx / V, c = idx % V;
        v[u] = (idx < total && x0 + c < ncols) ? src[(size_t)(r0 + i) * ld + x0 + c] : make_float2(0.f, 0.f);
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int idx = base + u * blockDim.x;
        if (idx < total) tile[(idx % V) * LEN + pad_idx(dst(r0 + idx / V))] = v[u];
      }
    }
  }
}

// Per-kernel launch facts, computed once per (kernel, device): the
// shared-memory opt-in and the resident CTAs per SM.  Kept off the per-launch
// path, which otherwise pays a driver query on every launch.
struct KernelFacts {
  int occ = 0;  // CTAs per SM (0 = not yet known)
  cudaError_t err = cudaSuccess;
};

// registry keyed by (kernel address, device); defined in capi.cu
KernelFacts& kernel_facts_slot(const void* kernel, int device);

template <class K>
inline KernelFacts& kernel_facts(K kernel, int threads, size_t smem) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) dev = 0;
  KernelFacts& f = kernel_facts_slot(reinterpret_cast<const void*>(kernel), dev);
  if (f.occ == 0) {
    if (smem > 48 * 1024) f.err = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int occ = 0;
    if (f.err == cudaSuccess &&
        (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, threads, smem) != cudaSuccess || occ < 1))
      occ = 1;
    f.occ = occ;
  }
  return f;
}

template <class K>
inline int persistent_grid(K kernel, int threads, size_t smem, long work_items_ctas) {
  KernelFacts& f = kernel_facts(kernel, threads, smem);
  long g = (long)sm_count() * f.occ;
  if (work_items_ctas < g) g = work_items_ctas;
  if (g < 1) g = 1;
  return (int)g;
}

template <class K>
inline cudaError_t set_smem(K kernel, size_t smem) {
  (void)kernel;
  (void)smem;
  return cudaSuccess;  // done once by kernel_facts (called by persistent_grid before every launch)
}

}  // namespace cx
