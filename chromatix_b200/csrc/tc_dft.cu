// Batched complex DFT on the tensor cores, split FP16 precision.
//
// A length-R complex DFT of 128 vectors is one real GEMM
//   D (128 x 2R) = A (128 x 2R) B (2R x 2R),
// A = the vectors' (re | im), B = [[Fr, Fi], [-Fi, Fr]] with F = exp(-+2 pi i n k / R).
// FP32 values are carried as FP16 hi + lo pairs (hi = fp16(x), lo =
// fp16(x - hi)); D = Ahi Bhi + Alo Bhi + Ahi Blo accumulates in FP32 in
// tensor memory (the lo * lo term, ~2^-22 relative, is dropped).  Each vector
// is scaled by a power of two (exact) so its largest component sits near
// 2^10, keeping hi and lo inside FP16's normal range.
//
// This is the building block of the split-precision transform stages: the
// radix-R butterflies of a Stockham / four-step FFT as dense contractions.
#include <cmath>

#include "host.cuh"
#include "tcgen05.cuh"

namespace cx {

template <int R>
struct TcDftCfg {
  static constexpr int M = 128;                       // vectors per MMA tile (one per thread)
  static constexpr int K = 2 * R;                     // (re | im) of the inputs
  static constexpr int KP = (K + 15) / 16 * 16;       // K padded to the MMA's K step
  static constexpr int NP = (2 * R + 15) / 16 * 16;   // outputs (re | im), N % 16 == 0 for M = 128
  static constexpr uint32_t A_BYTES = M * KP * 2;     // one of hi / lo
  static constexpr uint32_t B_BYTES = NP * KP * 2;
  static constexpr int TMEM_COLS = NP <= 32 ? 32 : NP <= 64 ? 64 : NP <= 128 ? 128 : 256;
  static constexpr size_t SMEM = 2 * (size_t)A_BYTES + 2 * (size_t)B_BYTES + 64;
  static constexpr int POLLS = 1 << 16;
};

// status_dev[0] is set to 1 if an MMA completion wait ran out (the tile is skipped)
template <int R>
__global__ void __launch_bounds__(128, 1) k_dft_split16(const float2* __restrict__ x, float2* __restrict__ y,
                                                         long batch, int inverse, int* status) {
  using C = TcDftCfg<R>;
  extern __shared__ __align__(128) uint8_t smem[];
  uint8_t* Ahi = smem;
  uint8_t* Alo = Ahi + C::A_BYTES;
  uint8_t* Bhi = Alo + C::A_BYTES;
  uint8_t* Blo = Bhi + C::B_BYTES;
  uint64_t* bar = reinterpret_cast<uint64_t*>(Blo + C::B_BYTES);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 1);
  const int tid = threadIdx.x, warp = tid >> 5;

  // B = the real-expanded DFT matrix, K-major (row j = output, column k = input)
  const double sgn = inverse ? 1.0 : -1.0;
  for (int idx = tid; idx < C::NP * C::KP; idx += blockDim.x) {
    const int j = idx / C::KP, k = idx % C::KP;
    float v = 0.f;
    if (j < 2 * R && k < 2 * R) {
      const int n = k % R, kk = j % R, pin = k / R, pout = j / R;
      double sd, cd;
      sincospi(sgn * 2.0 * (double)((n * kk) % R) / (double)R, &sd, &cd);
      // out_re = Fr in_re - Fi in_im ; out_im = Fi in_re + Fr in_im
      v = (float)(pin == pout ? cd : (pin == 0 ? sd : -sd));
    }
    const __half h = __float2half_rn(v);
    const __half l = __float2half_rn(v - __half2float(h));
    *reinterpret_cast<__half*>(Bhi + tc::off_kmajor(C::NP, j, k)) = h;
    *reinterpret_cast<__half*>(Blo + tc::off_kmajor(C::NP, j, k)) = l;
  }
  if (warp == 0) {
    tc::tmem_alloc(tslot, C::TMEM_COLS);
    tc::tmem_relinquish();
  }
  if (tid == 0) {
    tc::mbar_init(bar, 1);
    tc::mbar_init_fence();
  }
  tc::fence_smem_to_async();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tslot;
  constexpr uint32_t idesc = tc::idesc_f16_f32(C::M, C::NP, 0, 0);
  uint32_t phase = 0;
  bool failed = false;

  for (long tile = blockIdx.x; tile * C::M < batch; tile += gridDim.x) {
    const long v = tile * C::M + tid;
    const bool valid = v < batch;
    float2 xv[R];
    float mx = 0.f;
#pragma unroll
    for (int n = 0; n < R; ++n) {
      xv[n] = valid ? x[v * R + n] : make_float2(0.f, 0.f);
      mx = fmaxf(mx, fmaxf(fabsf(xv[n].x), fabsf(xv[n].y)));
    }
    // power-of-two scale: largest component near 2^10 (exact, undone on output)
    int e = 0;
    if (mx > 0.f) frexpf(mx, &e);
    const float sc = ldexpf(1.f, 10 - e), isc = ldexpf(1.f, e - 10);
    // A row `tid` (K-major): k < R re, R <= k < 2R im, zero beyond
#pragma unroll
    for (int kb = 0; kb < C::KP / 8; ++kb) {
      uint32_t hi[4], lo[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        float a2[2];
#pragma unroll
        for (int t = 0; t < 2; ++t) {
          const int k = kb * 8 + 2 * q + t;  // compile-time after unrolling
          a2[t] = 0.f;
          if (k < R)
            a2[t] = xv[k % R].x * sc;
          else if (k < 2 * R)
            a2[t] = xv[k % R].y * sc;
        }
        tc::split2(a2[0], a2[1], hi[q], lo[q]);
      }
      const uint32_t off = tc::off_kmajor(C::M, tid, kb * 8);
      *reinterpret_cast<uint4*>(Ahi + off) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
      *reinterpret_cast<uint4*>(Alo + off) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
    }
    tc::fence_smem_to_async();
    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
      const uint32_t a_lbo = (C::M / 8) * 128, b_lbo = (C::NP / 8) * 128;
#pragma unroll
      for (int s = 0; s < C::KP / 16; ++s) {
        const uint64_t ah = tc::smem_desc(tc::smem_u32(Ahi) + s * 2 * a_lbo, a_lbo, 128);
        const uint64_t al = tc::smem_desc(tc::smem_u32(Alo) + s * 2 * a_lbo, a_lbo, 128);
        const uint64_t bh = tc::smem_desc(tc::smem_u32(Bhi) + s * 2 * b_lbo, b_lbo, 128);
        const uint64_t bl = tc::smem_desc(tc::smem_u32(Blo) + s * 2 * b_lbo, b_lbo, 128);
        tc::mma_f16(tmem, ah, bh, idesc, s > 0 ? 1u : 0u);
        tc::mma_f16(tmem, al, bh, idesc, 1u);
        tc::mma_f16(tmem, ah, bl, idesc, 1u);
      }
      tc::mma_commit(bar);
    }
    const bool ok = tc::mbar_wait(bar, phase, C::POLLS);
    phase ^= 1u;
    if (!__syncthreads_and(ok)) {
      failed = true;
      break;
    }
    tc::fence_after_sync();
    float d[C::NP];
#pragma unroll
    for (int c = 0; c < C::NP; c += 16) tc::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + c, d + c);
    tc::tmem_wait_ld();
    if (valid) {
#pragma unroll
      for (int k = 0; k < R; ++k) y[v * R + k] = make_float2(d[k] * isc, d[R + k] * isc);
    }
    tc::fence_before_sync();
    __syncthreads();
  }
  if (failed) {
    if (tid == 0) atomicExch(status, 1);
    // let the MMAs in flight finish (bounded) before the tensor memory is freed
    tc::mbar_wait(bar, phase ^ 1u, C::POLLS);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, C::TMEM_COLS);
}

template <int R>
static cx_status launch_dft_split16(const float2* x, float2* y, long batch, int inverse, int* status,
                                    cudaStream_t st) {
  using C = TcDftCfg<R>;
  auto k = k_dft_split16<R>;
  CX_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM));
  long tiles = (batch + C::M - 1) / C::M;
  int grid = (int)(tiles < (long)sm_count() ? tiles : (long)sm_count());
  k<<<grid, 128, C::SMEM, st>>>(x, y, batch, inverse, status);
  CX_LAUNCH_CHECK();
  return CX_OK;
}

}  // namespace cx

using namespace cx;

extern "C" cx_status cx_dft_split16(const void* x, void* y, int32_t R, int64_t batch, int32_t inverse,
                                    int32_t* status_dev, cx_stream_t stream) {
  if (!x || !y || !status_dev || batch < 0) {
    set_error("cx_dft_split16: invalid arguments");
    return CX_ERR_INVALID;
  }
  if (batch == 0) return CX_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const float2* xi = static_cast<const float2*>(x);
  float2* yo = static_cast<float2*>(y);
  switch (R) {
    case 16: return launch_dft_split16<16>(xi, yo, batch, inverse, status_dev, st);
    case 32: return launch_dft_split16<32>(xi, yo, batch, inverse, status_dev, st);
    case 40: return launch_dft_split16<40>(xi, yo, batch, inverse, status_dev, st);
    case 64: return launch_dft_split16<64>(xi, yo, batch, inverse, status_dev, st);
    default: break;
  }
  set_error("cx_dft_split16: length %d not compiled in (16, 32, 40, 64)", R);
  return CX_ERR_UNSUPPORTED;
}
