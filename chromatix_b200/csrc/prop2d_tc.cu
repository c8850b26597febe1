// Column pass of the Fourier-multiplier propagation with the column FFTs on
// the tensor cores (CX_PREC_SPLIT16): per (output plane, eight-column tile)
// the four-step split-precision transform, x H(ky, kx) evaluated on the fly
// (the accurate-mode propagator of prop2d.cuh), and the inverse transform
// (tc_fft_mult_tile), writing only the output rows -- k_prop_cols with the
// radix butterflies replaced by dense DFT contractions.  In place when T == T2
// (the multislice slice loop): a tile is read completely before it is written.
#include "prop2d.cuh"
#include "tc_fft.cuh"

namespace cx {

// X H(ky, kx) out of line: the propagator's branches (kernel kinds, FP64
// phase) inlined at each of a tile's unrolled bins would overflow the
// instruction cache
__device__ __noinline__ float2 prop_mult(float2 X, int ky, int kx, const Prop2DArgs* a, const cx_plane* pl,
                                         const PropK* c) {
  return cmul(X, prop_kernel_k(ky, kx, *a, *pl, *c));
}

template <int N1, int N2>
struct PropTcCfg {
  using F = TcFft<N1, N2>;
  static constexpr int N = F::N;
  static constexpr size_t TW_BYTES = sizeof(float2) * N;
  static constexpr size_t SMEM = F::SMEM + TW_BYTES + 64 + 256;
};

template <int N1, int N2>
__global__ void __launch_bounds__(256, 1) k_prop_cols_tc(const float2* T, float2* T2, Prop2DArgs a,
                                                         const float2* __restrict__ twN, TcMats mats) {
  using F = TcFft<N1, N2>;
  using C = PropTcCfg<N1, N2>;
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

  const int tiles_x = a.px / 8;
  const long total = (long)tiles_x * a.n_out_planes;
  const float scale = 1.0f / ((float)a.py * (float)a.px);
  long t = blockIdx.x;
  for (; t < total; t += gridDim.x) {
    const int q = (int)(t / tiles_x);
    const int x0 = (int)(t % tiles_x) * 8;
    const cx_plane pl = a.planes[q];
    const float2* src = T + (size_t)pl.in_plane * a.ny * a.px + x0;
    float2* dst = T2 + (size_t)q * a.out_ny * a.px + x0;
    auto load8 = [&](int n, int v, float2* o) {
      // column v of padded-grid rows n .. n+7; row n holds data row n - pad_y
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int r = n + j - a.pad_y;
        o[j] = (r >= 0 && r < a.ny) ? src[(size_t)r * a.px + v] : make_float2(0.f, 0.f);
      }
    };
    const PropK kc = prop_consts(a, pl);
    auto mult = [&](int k, int v, float2 X) { return prop_mult(X, k, x0 + v, &a, &pl, &kc); };
    auto store_row = [&](int n, const float2* row) {
      const int r = n - a.out_y0;
      if (r >= 0 && r < a.out_ny) {
        float4* p = reinterpret_cast<float4*>(dst + (size_t)r * a.px);
#pragma unroll
        for (int k = 0; k < 4; ++k)
          p[k] = make_float4(row[2 * k].x * scale, row[2 * k].y * scale, row[2 * k + 1].x * scale,
                             row[2 * k + 1].y * scale);
      }
    };
    if (!tc_fft_mult_tile<F>(S, tmem, phase, tw, load8, mult, store_row)) {
      failed = true;
      break;
    }
  }
  if (failed) {
    // an MMA wait ran out: mark this CTA's unfinished output tiles invalid
    // (NaN) and let the MMAs in flight finish (bounded) before freeing tensor memory
    tc::mbar_wait(S.bar, phase ^ 1u, F::POLLS);
    tc_note_timeout(mats);
    const float nan = __int_as_float(0x7fc00000);
    for (; t < total; t += gridDim.x) {
      const int q = (int)(t / tiles_x), x0 = (int)(t % tiles_x) * 8;
      float2* dst = T2 + (size_t)q * a.out_ny * a.px + x0;
      for (int idx = tid; idx < a.out_ny * 8; idx += blockDim.x) dst[(size_t)(idx >> 3) * a.px + (idx & 7)] =
          make_float2(nan, nan);
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if ((tid >> 5) == 0) tc::tmem_dealloc(tmem, F::TMEM_COLS);
}

template <int N1, int N2>
static cx_status launch_prop_cols_tc(const float2* T, float2* T2, const Prop2DArgs& a, cudaStream_t st) {
  using C = PropTcCfg<N1, N2>;
  auto k = k_prop_cols_tc<N1, N2>;
  CX_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM));
  const long items = (long)(a.px / 8) * a.n_out_planes;
  int grid = sm_count();
  if (items < grid) grid = (int)items;
  TcMats mats;
  if (const cx_status e = tc_mats(N1, N2, &mats)) return e;
  k<<<grid, 256, C::SMEM, st>>>(T, T2, a, a.twg + tw_offset(C::N), mats);
  CX_LAUNCH_CHECK();
  return CX_OK;
}

// Row passes with the row FFTs on the tensor cores (tc_fft_rows_tile), eight
// rows per tile.  INV = false: k_prop_rows_fwd (the data rows of every input
// plane, zero padding along x in the loader); INV = true: k_prop_rows_inv
// (the output rows, inverse transform as conj(FFT(conj .)), crop in the store).
struct PropTcRow {
  const float2* src;
  float2* dst;
  int valid, pad;
};

template <int N1, int N2>
struct PropTcRowCfg {
  using F = TcFft<N1, N2>;
  static constexpr int N = F::N;
  static constexpr size_t TW_BYTES = sizeof(float2) * N;
  static constexpr size_t SMEM = F::SMEM + TW_BYTES + 64 + 256 + 8 * sizeof(PropTcRow);
};

template <int N1, int N2, bool INV>
__global__ void __launch_bounds__(256, 1) k_prop_rows_tc(const float2* in, float2* out, Prop2DArgs a,
                                                         const float2* __restrict__ twN, TcMats mats) {
  using F = TcFft<N1, N2>;
  using C = PropTcRowCfg<N1, N2>;
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
  PropTcRow* rp = reinterpret_cast<PropTcRow*>(S.red + 64);
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

  const int rows = INV ? a.out_ny : a.ny;
  const long total = (long)(INV ? a.n_out_planes : a.n_in_planes) * rows;
  const long tiles = (total + 7) / 8;
  const int W = a.W;
  for (long t = blockIdx.x; t < tiles; t += gridDim.x) {
    if (tid < 8) {
      const long item = t * 8 + tid;
      const bool valid = item < total;
      const int p = valid ? (int)(item / rows) : 0;
      const int y = valid ? (int)(item % rows) : 0;
      const int b = p / W, w = p % W;
      PropTcRow r;
      if (!INV) {
        const float2* ub = a.in_ptrs ? a.in_ptrs[b] : in + (size_t)b * a.ny * a.nx * W;
        r.src = ub + (size_t)y * a.nx * W + w;
        r.dst = out + ((size_t)p * a.ny + y) * a.px;
      } else {
        float2* ob = a.out_ptrs ? a.out_ptrs[b] : out + (size_t)b * a.out_ny * a.out_nx * W;
        r.src = in + ((size_t)p * a.out_ny + y) * a.px;
        r.dst = ob + (size_t)y * a.out_nx * W + w;
      }
      r.valid = valid ? 1 : 0;
      r.pad = 0;
      rp[tid] = r;
    }
    __syncthreads();
    auto load8 = [&](int v, int n, float2* o) {
      const PropTcRow& r = rp[v];
      if (!INV) {
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int x = n + q - a.pad_x;
          o[q] = (r.valid && x >= 0 && x < a.nx) ? r.src[(size_t)x * W] : make_float2(0.f, 0.f);
        }
      } else if (r.valid) {
        const float4* s4 = reinterpret_cast<const float4*>(r.src + n);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const float4 f = s4[k];
          o[2 * k] = make_float2(f.x, -f.y);
          o[2 * k + 1] = make_float2(f.z, -f.w);
        }
      } else {
#pragma unroll
        for (int q = 0; q < 8; ++q) o[q] = make_float2(0.f, 0.f);
      }
    };
    auto store = [&](int v, int k, float2 X) {
      const PropTcRow& r = rp[v];
      if (!r.valid) return;
      if (!INV) {
        r.dst[k] = X;
      } else {
        const int x = k - a.out_x0;
        if (x >= 0 && x < a.out_nx) r.dst[(size_t)x * W] = make_float2(X.x, -X.y);
      }
    };
    if (!tc_fft_rows_tile<F>(S, tmem, phase, tw, load8, store)) {
      // an MMA wait ran out: mark this CTA's remaining rows invalid (NaN) and
      // let the MMAs in flight finish (bounded) before tensor memory is freed
      tc::mbar_wait(S.bar, phase ^ 1u, F::POLLS);
      tc_note_timeout(mats);
      const float nan = __int_as_float(0x7fc00000);
      for (long u = t; u < tiles; u += gridDim.x) {
        for (int idx = tid; idx < 8 * N; idx += blockDim.x) {
          const long item = u * 8 + idx / N;
          if (item >= total) continue;
          const int p = (int)(item / rows), y = (int)(item % rows), k = idx % N;
          const int b = p / W, w = p % W;
          if (!INV) {
            out[((size_t)p * a.ny + y) * a.px + k] = make_float2(nan, nan);
          } else {
            const int x = k - a.out_x0;
            float2* ob = a.out_ptrs ? a.out_ptrs[b] : out + (size_t)b * a.out_ny * a.out_nx * W;
            if (x >= 0 && x < a.out_nx) ob[((size_t)y * a.out_nx + x) * W + w] = make_float2(nan, nan);
          }
        }
      }
      break;
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if ((tid >> 5) == 0) tc::tmem_dealloc(tmem, F::TMEM_COLS);
}

template <int N1, int N2, bool INV>
static cx_status launch_prop_rows_tc(const float2* in, float2* out, const Prop2DArgs& a, cudaStream_t st) {
  using C = PropTcRowCfg<N1, N2>;
  auto k = k_prop_rows_tc<N1, N2, INV>;
  CX_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM));
  const long tiles = ((long)(INV ? a.n_out_planes : a.n_in_planes) * (INV ? a.out_ny : a.ny) + 7) / 8;
  int grid = sm_count();
  if (tiles < grid) grid = (int)tiles;
  TcMats mats;
  if (const cx_status e = tc_mats(N1, N2, &mats)) return e;
  k<<<grid, 256, C::SMEM, st>>>(in, out, a, a.twg + tw_offset(C::N), mats);
  CX_LAUNCH_CHECK();
  return CX_OK;
}

bool prop_tc_rows_supported(int px) { return px == 1024 || px == 1280; }

cx_status dispatch_rows_tc(bool inverse, const float2* in, float2* out, const Prop2DArgs& a, cudaStream_t st) {
  if (!prop_tc_rows_supported(a.px)) {
    set_error("split-precision row pass: %d padded columns not compiled in (1024 or 1280)", a.px);
    return CX_ERR_UNSUPPORTED;
  }
  if (a.px == 1280)
    return inverse ? launch_prop_rows_tc<40, 32, true>(in, out, a, st) : launch_prop_rows_tc<40, 32, false>(in, out, a, st);
  return inverse ? launch_prop_rows_tc<32, 32, true>(in, out, a, st) : launch_prop_rows_tc<32, 32, false>(in, out, a, st);
}

bool prop_tc_supported(int py, int px) { return (py == 1024 || py == 1280) && px % 8 == 0 && px >= 8; }

cx_status dispatch_cols_tc(int n, const float2* T, float2* T2, const Prop2DArgs& a, cudaStream_t st) {
  if (!prop_tc_supported(n, a.px)) {
    set_error("split-precision column pass: padded grid %dx%d not compiled in (1024 or 1280 rows, columns a "
              "multiple of 8)", n, a.px);
    return CX_ERR_UNSUPPORTED;
  }
  return n == 1280 ? launch_prop_cols_tc<40, 32>(T, T2, a, st) : launch_prop_cols_tc<32, 32>(T, T2, a, st);
}

}  // namespace cx
