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
__global__ void __launch_bounds__(256, 1) k_psf_cols_tc(PsfArgs a, const float2* __restrict__ twN, TcMats mats) {
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

  tc_fft_copy_b(S.B1, mats.b1, F::B1_BYTES, tid, blockDim.x);
  tc_fft_copy_b(S.B2, mats.b2, F::B2_BYTES, tid, blockDim.x);
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
      // the pupil's support have a zero spectrum; column v of rows n .. n+7
      auto load8 = [&](int n, int v, float2* o) {
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int y = add_mod(n + j, N / 2, N);
          o[j] = (y >= slo && y < shi) ? src[(size_t)(y - ylo) * a.nx + v] : make_float2(0.f, 0.f);
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
    tc_note_timeout(mats);
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
  TcMats mats;
  if (const cx_status e = tc_mats(N1, N2, &mats)) return e;
  k<<<grid, 256, C::SMEM, st>>>(a, a.twg + tw_offset(C::N), mats);
  CX_LAUNCH_CHECK();
  return CX_OK;
}

// Row pass with the row FFTs on the tensor cores: eight row spectra per tile
// (consecutive items (z, compact row) as in k_psf_rows_tab), the table source
// M * CX * row factor evaluated in the loader (ifftshift along x), the
// four-step row transform of tc_fft_rows_tile, the row spectrum stored for
// live rows only (rows outside the pupil transform zeros and store nothing).
struct PsfTcRow {
  const float2* mrow;
  const float2* cxz;
  float2* dst;
  float2 cy;
  int xlo, nc, live, pad;
};

template <int N1, int N2>
struct PsfTcRowCfg {
  using F = TcFft<N1, N2>;
  static constexpr int N = F::N;
  static constexpr size_t TW_BYTES = sizeof(float2) * N;
  static constexpr size_t SMEM = F::SMEM + TW_BYTES + 64 + 256 + 8 * sizeof(PsfTcRow);
};

template <int N1, int N2>
__global__ void __launch_bounds__(256, 1) k_psf_rows_tc(PsfArgs a, const float2* __restrict__ twN, TcMats mats) {
  using F = TcFft<N1, N2>;
  using C = PsfTcRowCfg<N1, N2>;
  constexpr int N = F::N;
  extern __shared__ __align__(128) uint8_t smem[];
  TcFftSmem S;
  S.A = smem;
  S.B1 = smem + F::A_BYTES;
  S.B2 = S.B1 + F::B1_BYTES;
  float2* tw = reinterpret_cast<float2*>(S.B2 + F::B2_BYTES);
  S.bar = reinterpret_cast<uint64_t*>(reinterpret_cast<uint8_t*>(tw) + C::TW_BYTES);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(S.bar + 1);
  S.red = reinterpret_cast<float*>(S.bar + 8);
  PsfTcRow* rp = reinterpret_cast<PsfTcRow*>(S.red + 64);
  const int tid = threadIdx.x;

  tc_fft_copy_b(S.B1, mats.b1, F::B1_BYTES, tid, blockDim.x);
  tc_fft_copy_b(S.B2, mats.b2, F::B2_BYTES, tid, blockDim.x);
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

  const long total = (long)a.zc * a.rowsum;
  const long tiles = (total + 7) / 8;
  const double PI = 3.141592653589793238462643383279502884;
  for (long t = blockIdx.x; t < tiles; t += gridDim.x) {
    if (tid < 8) {
      const long item0 = t * 8 + tid;
      const long item = item0 < total ? item0 : total - 1;
      const int zl = (int)(item / a.rowsum);
      const int rem = (int)(item % a.rowsum);
      int w = 0;
      while (w + 1 < a.W && rem >= a.prefix[w + 1]) ++w;
      const PsfWv& p = a.wv[w];
      const int y = a.ylo[w] + (rem - a.prefix[w]);
      const bool live = item0 < total && y >= support_lo(a, w) && y < support_hi(a, w);
      const double z = a.z[a.z0 + zl];
      const double gyo = p.dy * ((double)y - (double)a.ny * 0.5) - a.offy;
      const double qz = -PI * (z / a.f_obj) / p.L2;
      PsfTcRow r;
      r.mrow = a.M + a.mprefix[w] + (size_t)(y - a.ylo[w]) * a.ncols[w];
      r.cxz = a.CX + (size_t)(a.z0 + zl) * a.csum + a.cprefix[w];
      r.dst = a.T + ((size_t)zl * a.rowsum + rem) * a.nx;
      r.cy = expi_precise(qz * gyo * gyo);
      r.xlo = a.xlo[w];
      r.nc = live ? a.ncols[w] : 0;
      r.live = live ? 1 : 0;
      r.pad = 0;
      rp[tid] = r;
    }
    __syncthreads();
    auto load8 = [&](int v, int n, float2* o) {
      const PsfTcRow& r = rp[v];
      // ifftshift along x: eight consecutive FFT inputs are eight consecutive
      // field columns (N / 2 and n are multiples of 8), then the box column
      const int c0 = add_mod(n, N / 2, N) - r.xlo;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int c = c0 + q;
        o[q] = (unsigned)c < (unsigned)r.nc ? cmul(cmul(r.mrow[c], r.cxz[c]), r.cy) : make_float2(0.f, 0.f);
      }
    };
    auto store = [&](int v, int k, float2 X) {
      if (rp[v].live) rp[v].dst[k] = X;
    };
    if (!tc_fft_rows_tile<F>(S, tmem, phase, tw, load8, store)) {
      // an MMA wait ran out: mark this CTA's remaining row spectra invalid
      // (NaN; the column pass carries them into the intensity) and let the
      // MMAs in flight finish (bounded) before tensor memory is freed
      tc::mbar_wait(S.bar, phase ^ 1u, F::POLLS);
      tc_note_timeout(mats);
      const float nan = __int_as_float(0x7fc00000);
      for (long u = t; u < tiles; u += gridDim.x)
        for (int idx = tid; idx < 8 * N; idx += blockDim.x) {
          const long item = u * 8 + idx / N;
          if (item < total) a.T[item * a.nx + idx % N] = make_float2(nan, nan);
        }
      break;
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if ((tid >> 5) == 0) tc::tmem_dealloc(tmem, F::TMEM_COLS);
}

template <int N1, int N2>
static cx_status launch_psf_rows_tc(const PsfArgs& a, cudaStream_t st) {
  using C = PsfTcRowCfg<N1, N2>;
  auto k = k_psf_rows_tc<N1, N2>;
  CX_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM));
  const long tiles = ((long)a.zc * a.rowsum + 7) / 8;
  int grid = sm_count();
  if (tiles < grid) grid = (int)tiles;
  TcMats mats;
  if (const cx_status e = tc_mats(N1, N2, &mats)) return e;
  k<<<grid, 256, C::SMEM, st>>>(a, a.twg + tw_offset(C::N), mats);
  CX_LAUNCH_CHECK();
  return CX_OK;
}

bool psf_tc_rows_supported(int nx) { return nx == 1280 || nx == 1024; }

cx_status psf_dispatch_rows_tc(int n, const PsfArgs& a, cudaStream_t st) {
  if (!psf_tc_rows_supported(n)) {
    set_error("split-precision PSF row pass: %d columns not compiled in (1024 or 1280)", n);
    return CX_ERR_UNSUPPORTED;
  }
  return n == 1280 ? launch_psf_rows_tc<40, 32>(a, st) : launch_psf_rows_tc<32, 32>(a, st);
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
