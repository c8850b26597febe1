// Column pass of the fused PSF with the column FFTs on the tensor cores
// (CX_PREC_SPLIT16): per (z, eight-column tile) and wavelength, the four-step
// split-precision transform of tc_fft.cuh over the tile of row spectra, the
// spectral intensity density * |X|^2 accumulated in shared memory, and the
// fftshifted intensity stored once -- the same pass as k_psf_cols with the
// radix butterflies replaced by dense DFT contractions.
#include "psf.cuh"
#include "tc_fft.cuh"

namespace cx {

template <int N1, int N2>
struct PsfTcCfg {
  using F = TcFft<N1, N2>;
  static constexpr int N = F::N, ACC = N + 1;  // odd float stride per column
  static constexpr size_t ACC_BYTES = sizeof(float) * 8 * ACC;
  static constexpr size_t TW_BYTES = sizeof(float2) * N;
  static constexpr size_t SMEM = F::SMEM + ((ACC_BYTES + 15) & ~(size_t)15) + TW_BYTES + 64 + 256;
};

template <int N1, int N2>
__global__ void __launch_bounds__(256, 1) k_psf_cols_tc(PsfArgs a, const float2* __restrict__ twN) {
  using F = TcFft<N1, N2>;
  using C = PsfTcCfg<N1, N2>;
  constexpr int N = F::N, ACC = C::ACC;
  extern __shared__ __align__(128) uint8_t smem[];
  TcFftSmem S;
  S.A = smem;
  S.B1 = smem + F::A_BYTES;
  S.B2 = S.B1 + F::B1_BYTES;
  float* acc = reinterpret_cast<float*>(S.B2 + F::B2_BYTES);
  float2* tw = reinterpret_cast<float2*>(reinterpret_cast<uint8_t*>(acc) + ((C::ACC_BYTES + 15) & ~(size_t)15));
  S.bar = reinterpret_cast<uint64_t*>(reinterpret_cast<uint8_t*>(tw) + C::TW_BYTES);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(S.bar + 1);
  S.red = reinterpret_cast<float*>(S.bar + 8);
  const int tid = threadIdx.x;

  tc_fft_build_b<N1>(S.B1, false, tid, blockDim.x);
  tc_fft_build_b<N2>(S.B2, false, tid, blockDim.x);
  for (int i = tid; i < N; i += blockDim.x) tw[i] = twN[i];
  if ((tid >> 5) == 0) {
    tc::tmem_alloc(tslot, F::TMEM_COLS);
    tc::tmem_relinquish();
  }
  if (tid == 0) {
    tc::mbar_init(S.bar, 1);
    tc::mbar_init_fence();
  }
  tc::fence_smem_to_async();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tslot;
  uint32_t phase = 0;
  bool failed = false;

  const int tiles_x = a.nx / 8;
  const long total = (long)tiles_x * a.zc;
  for (long t = blockIdx.x; t < total && !failed; t += gridDim.x) {
    const int zl = (int)(t / tiles_x);
    const int x0 = (int)(t % tiles_x) * 8;
    for (int w = 0; w < a.W && !failed; ++w) {
      const PsfWv& p = a.wv[w];
      const float dens = (float)p.dens;
      const float2* src = a.T + ((size_t)zl * a.rowsum + a.prefix[w]) * a.nx + x0;
      const int ylo = a.ylo[w], slo = support_lo(a, w), shi = support_hi(a, w);
      // FFT row n holds field row (n + N/2) mod N (ifftshift); rows outside
      // the pupil's support have a zero spectrum
      auto load8 = [&](int n, float2* o) {
        const int y = add_mod(n, N / 2, N);
        if (y >= slo && y < shi) {
          const float4* r = reinterpret_cast<const float4*>(src + (size_t)(y - ylo) * a.nx);
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const float4 f = r[q];
            o[2 * q] = make_float2(f.x, f.y);
            o[2 * q + 1] = make_float2(f.z, f.w);
          }
        } else {
#pragma unroll
          for (int q = 0; q < 8; ++q) o[q] = make_float2(0.f, 0.f);
        }
      };
      auto store = [&](int k, int v, float2 X) {
        const float e = dens * cabs2(X);
        acc[v * ACC + k] = (w == 0) ? e : acc[v * ACC + k] + e;
      };
      if (!tc_fft_tile<F>(S, tmem, phase, tw, false, load8, store)) failed = true;
    }
    if (failed) break;
    __syncthreads();
    float* outz = a.out + (size_t)(a.z0 + zl) * a.ny * a.nx;
    for (int idx = tid; idx < N * 8; idx += blockDim.x) {
      const int row = idx >> 3, c = idx & 7;
      const int k = add_mod(row, N - N / 2, N);  // fftshift along y
      outz[(size_t)row * a.nx + add_mod(x0 + c, a.nx / 2, a.nx)] = acc[c * ACC + k];
    }
    __syncthreads();
  }
  if (failed) {
    // an MMA wait ran out: mark this CTA's remaining output as invalid (NaN),
    // let the MMAs in flight finish (bounded) before the tensor memory is freed
    tc::mbar_wait(S.bar, phase ^ 1u, F::POLLS);
    for (long t = blockIdx.x; t < total; t += gridDim.x) {
      const int zl = (int)(t / tiles_x), x0 = (int)(t % tiles_x) * 8;
      float* outz = a.out + (size_t)(a.z0 + zl) * a.ny * a.nx;
      for (int idx = tid; idx < N * 8; idx += blockDim.x)
        outz[(size_t)(idx >> 3) * a.nx + add_mod(x0 + (idx & 7), a.nx / 2, a.nx)] = __int_as_float(0x7fc00000);
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if ((tid >> 5) == 0) tc::tmem_dealloc(tmem, F::TMEM_COLS);
}

template <int N1, int N2>
static cx_status launch_psf_cols_tc(const PsfArgs& a, cudaStream_t st) {
  using C = PsfTcCfg<N1, N2>;
  auto k = k_psf_cols_tc<N1, N2>;
  CX_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM));
  const long items = (long)(a.nx / 8) * a.zc;
  int grid = sm_count();
  if (items < grid) grid = (int)items;
  k<<<grid, 256, C::SMEM, st>>>(a, a.twg + tw_offset(C::N));
  CX_LAUNCH_CHECK();
  return CX_OK;
}

bool psf_tc_supported(int ny, int nx) { return (ny == 1280 || ny == 1024) && nx % 8 == 0 && nx >= 8; }

cx_status psf_dispatch_cols_tc(int n, const PsfArgs& a, cudaStream_t st) {
  if (!psf_tc_supported(n, a.nx)) {
    set_error("split-precision PSF column pass: grid %dx%d not compiled in (ny 1024 or 1280, nx a multiple of 8)",
              n, a.nx);
    return CX_ERR_UNSUPPORTED;
  }
  return n == 1280 ? launch_psf_cols_tc<40, 32>(a, st) : launch_psf_cols_tc<32, 32>(a, st);
}

}  // namespace cx
