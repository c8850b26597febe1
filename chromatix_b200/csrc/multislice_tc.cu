// Row passes of the multislice loop with the row transforms on the tensor
// cores (CX_PREC_SPLIT16, padded rows of 1024 or 1280): eight rows per tile,
// k_ms_rows' modes with its team FFTs replaced by tc_fft_rows_tile.  The slice
// step's inverse transform is conj(FFT(conj .)) and leaves its rows in shared
// memory; the forward transform's loader reads them back, applies the
// thin-sample step (transmittance, record, or the adjoint's gradients and
// conj(t)) and the output row spectrum is written over the input rows.
#include "multislice.cuh"
#include "tc_fft.cuh"

namespace cx {

template <int N1, int N2>
struct MsTcCfg {
  using F = TcFft<N1, N2>;
  static constexpr int N = F::N;
  static constexpr size_t TW_BYTES = sizeof(float2) * N;
  static constexpr size_t SMEM = F::SMEM + TW_BYTES + 64 + 256;
};

template <int N1, int N2, int MODE>
__global__ void __launch_bounds__(256, 1) k_ms_rows_tc(MsArgs a, const float2* __restrict__ twN, TcMats mats) {
  using F = TcFft<N1, N2>;
  using C = MsTcCfg<N1, N2>;
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

  const int r0 = MODE == MS_FINAL ? a.pad_y : 0;
  const int nrows = MODE == MS_FINAL ? a.ny : a.py;
  const long tiles = (nrows + 7) / 8;
  const size_t plane_d = (size_t)a.slice * a.ny * a.nx;
  const double kdz = 6.283185307179586476925286766559 * a.dz / a.lam;
  auto nothing = [](int, int, float2) {};
  bool ok = true;
  long t = blockIdx.x;
  for (; t < tiles && ok; t += gridDim.x) {
    const int y0 = r0 + (int)t * 8;
    auto valid = [&](int v) { return y0 + v < r0 + nrows; };
    auto row = [&](int v) { return a.buf + (size_t)(y0 + v) * a.px; };
    // inverse transform input: conj(row)
    auto load_conj = [&](int v, int n, float2* o) {
      if (valid(v)) {
        const float4* p = reinterpret_cast<const float4*>(row(v) + n);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const float4 f = p[k];
          o[2 * k] = make_float2(f.x, -f.y);
          o[2 * k + 1] = make_float2(f.z, -f.w);
        }
      } else {
#pragma unroll
        for (int q = 0; q < 8; ++q) o[q] = make_float2(0.f, 0.f);
      }
    };
    auto store_row = [&](int v, int k, float2 X) {
      if (valid(v)) row(v)[k] = X;
    };
    if constexpr (MODE == MS_LOAD) {
      auto load = [&](int v, int n, float2* o) {
        const int y = y0 + v, ys = y - a.oy;
        const bool rin = valid(v) && ys >= 0 && ys < a.sy;
        const float2* srow = a.src + (size_t)(rin ? ys : 0) * a.sx;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int xs = n + q - a.ox;
          o[q] = (rin && xs >= 0 && xs < a.sx) ? cscale(srow[xs], a.load_scale) : make_float2(0.f, 0.f);
          if (a.record && valid(v)) a.rec[(size_t)y * a.px + n + q] = o[q];
        }
      };
      ok = tc_fft_rows_tile<F>(S, tmem, phase, tw, load, store_row);
    } else if constexpr (MODE == MS_FINAL) {
      auto store = [&](int v, int k, float2 X) {
        const int xd = k - a.pad_x;
        if (valid(v) && xd >= 0 && xd < a.nx)
          a.dst[(size_t)(y0 + v - a.pad_y) * a.nx + xd] = make_float2(X.x, -X.y);
      };
      ok = tc_fft_rows_tile<F>(S, tmem, phase, tw, load_conj, store);
    } else {
      // inverse transform; its rows stay in shared memory as conj(IFFT(row))
      ok = tc_fft_rows_tile<F, false>(S, tmem, phase, tw, load_conj, nothing);
      if (!ok) break;
      const float2* stg = tc_rows_staged(S);
      auto load_step = [&](int v, int n, float2* o) {
        const int y = y0 + v, yd = y - a.pad_y;
        const bool yin = valid(v) && yd >= 0 && yd < a.ny;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int k = n + q, xd = k - a.pad_x;
          const float2 c = stg[v * N + k];
          float2 x = make_float2(c.x, -c.y);
          if (yin && xd >= 0 && xd < a.nx) {
            const size_t idx = plane_d + (size_t)yd * a.nx + xd;
            const float2 tr = ms_transmittance(a, a.dn[idx], a.ab[idx]);
            if constexpr (MODE == MS_FWD) {
              x = cmul(x, tr);
            } else {  // MS_BWD: x is g; w = g conj(u)
              const float2 u = a.rec_u[(size_t)y * a.px + k];
              const float wr = x.x * u.x + x.y * u.y, wi = x.y * u.x - x.x * u.y;
              const size_t gi = (size_t)yd * a.nx + xd;
              a.gdn[gi] = (float)(kdz * (double)wi);
              a.gab[gi] = (float)(-kdz * (double)wr);
              x = cmul(x, cconj(tr));
            }
          }
          if constexpr (MODE == MS_FWD) {
            if (a.record && valid(v)) a.rec[(size_t)y * a.px + k] = x;
          }
          o[q] = valid(v) ? x : make_float2(0.f, 0.f);
        }
      };
      ok = tc_fft_rows_tile<F>(S, tmem, phase, tw, load_step, store_row);
    }
  }
  if (!ok) {
    // an MMA wait ran out: mark the rows this CTA had not finished invalid
    // (NaN) and let the MMAs in flight finish (bounded) before tensor memory
    // is freed
    tc::mbar_wait(S.bar, phase ^ 1u, F::POLLS);
    tc_note_timeout(mats);
    const float nan = __int_as_float(0x7fc00000);
    for (long u = t; u < tiles; u += gridDim.x) {
      const int y0 = r0 + (int)u * 8;
      for (int idx = tid; idx < 8 * N; idx += blockDim.x) {
        const int v = idx / N, k = idx % N;
        if (y0 + v >= r0 + nrows) continue;
        if (MODE == MS_FINAL) {
          const int xd = k - a.pad_x;
          if (xd >= 0 && xd < a.nx) a.dst[(size_t)(y0 + v - a.pad_y) * a.nx + xd] = make_float2(nan, nan);
        } else {
          a.buf[(size_t)(y0 + v) * a.px + k] = make_float2(nan, nan);
        }
      }
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if ((tid >> 5) == 0) tc::tmem_dealloc(tmem, F::TMEM_COLS);
}

template <int N1, int N2, int MODE>
static cx_status launch_ms_rows_tc(const MsArgs& a, cudaStream_t st) {
  using C = MsTcCfg<N1, N2>;
  auto k = k_ms_rows_tc<N1, N2, MODE>;
  CX_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM));
  const long tiles = ((a.mode == MS_FINAL ? a.ny : a.py) + 7) / 8;
  int grid = sm_count();
  if (tiles < grid) grid = (int)tiles;
  TcMats mats;
  if (const cx_status e = tc_mats(N1, N2, &mats)) return e;
  k<<<grid, 256, C::SMEM, st>>>(a, a.twg + tw_offset(C::N), mats);
  CX_LAUNCH_CHECK();
  return CX_OK;
}

template <int N1, int N2>
static cx_status launch_ms_rows_tc_mode(const MsArgs& a, cudaStream_t st) {
  switch (a.mode) {
    case MS_LOAD:
      return launch_ms_rows_tc<N1, N2, MS_LOAD>(a, st);
    case MS_FWD:
      return launch_ms_rows_tc<N1, N2, MS_FWD>(a, st);
    case MS_BWD:
      return launch_ms_rows_tc<N1, N2, MS_BWD>(a, st);
    case MS_FINAL:
      return launch_ms_rows_tc<N1, N2, MS_FINAL>(a, st);
  }
  set_error("split-precision multislice row pass: mode %d has no tensor-core form", a.mode);
  return CX_ERR_UNSUPPORTED;
}

bool ms_tc_rows_supported(int px, int mode) { return (px == 1024 || px == 1280) && mode != MS_FLUOR; }

cx_status ms_dispatch_rows_tc(const MsArgs& a, cudaStream_t st) {
  if (!ms_tc_rows_supported(a.px, a.mode)) {
    set_error("split-precision multislice row pass: %d padded columns not compiled in (1024 or 1280)", a.px);
    return CX_ERR_UNSUPPORTED;
  }
  return a.px == 1280 ? launch_ms_rows_tc_mode<40, 32>(a, st) : launch_ms_rows_tc_mode<32, 32>(a, st);
}

}  // namespace cx
