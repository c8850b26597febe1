// Incoherent imaging: plane-wise 2D Fourier convolution of a sample stack with
// a PSF stack, summed over the planes by the sensor.
//
// Reference: ops/ops.py:9-86 (fourier_convolution: rfftn / irfftn at the next
// power of two of the summed shape, "same" crop from offset (k - 1) // 2),
// functional/sensors.py:85-86 (basic_sensor's sum over reduce_axis),
// systems/microscopes.py:271-297 (Microscope.image).
//
// Both inputs are real, so every transform is real-to-complex:
//   rows     r2c of length Q through a complex FFT of length M = Q/2 on
//            z[n] = x[2n] + i x[2n+1], then X[k] = E[k] + W^k O[k] with
//            E = (Z[k] + conj Z[M-k]) / 2, O = (Z[k] - conj Z[M-k]) / (2i),
//            W = exp(-2 pi i / Q), k = 0..M (NC = M + 1 spectrum columns)
//   columns  complex FFT of length P of the sample and the PSF column, the
//            product accumulated over the planes in registers, added once
//            per plane chunk into the transposed spectrum St (NC, P)
//   final    column inverse of St (rows of the crop kept), then per output
//            row the c2r of length Q through a complex inverse of length M:
//            Z'[k] = E[k] + i O[k], E = (Y[k] + conj Y[M-k]) / 2,
//            O = (Y[k] - conj Y[M-k]) W^-k / 2, x[2n] + i x[2n+1] = z'[n],
//            scaled by 2 / (P Q) (irfftn's 1 / (P Q) with the half-length
//            inverse), "same" crop from ((h-1)//2, (w-1)//2).
#pragma once
#include "host.cuh"

namespace cx {

// power-of-two transform lengths of the convolution (next_order of 2 h, 2 w)
#define CX_CONV_SIZES(X) X(2) X(4) X(8) X(16) X(32) X(64) X(128) X(256) X(512) X(1024) X(2048) X(4096)

struct ConvArgs {
  int h, w, P, Q, M, NC;  // image shape, transform lengths, M = Q / 2, NC = M + 1
  int z0, zc;             // plane chunk
  const float* a;         // sample (n_planes, h, w)
  const float* b;         // PSF (n_planes, h, w)
  float2* T;              // row spectra (zc, 2, h, NC)
  float2* St;             // accumulated spectrum, transposed (NC, P)
  float2* U;              // column inverse of the crop rows, transposed (NC, h)
  float* out;             // image (h, w)
  int c0y, c0x;           // "same" crop offsets
  float scale;            // 2 / (P Q)
  const float2* twg;
};

// ---------------------------------------------------------------------------
// rows: r2c of the zc planes of both stacks (items: plane, stack, row)
// ---------------------------------------------------------------------------
template <int M>
__global__ void __launch_bounds__(RowCfg<M>::THREADS, RowCfg<M>::MINB) k_conv_rows(ConvArgs a) {
  using C = RowCfg<M>;
  constexpr int QN = 2 * M;
  extern __shared__ float2 sm[];
  float2* tw = sm;
  load_twiddles<M>(tw, a.twg, threadIdx.x, blockDim.x);
  __syncthreads();
  constexpr int OFF_Q = tw_offset(QN);
  const float2* wq = a.twg + OFF_Q;  // exp(-2 pi i k / Q), k < Q
  const int team = threadIdx.x / C::LPV, lane = threadIdx.x % C::LPV;
  float2* s = sm + C::TW + team * Plan<M>::LEN;
  const long total = (long)a.zc * 2 * a.h;
  for (long base = (long)blockIdx.x * C::TEAMS; base < total; base += (long)gridDim.x * C::TEAMS) {
    const long item = base + team;
    if (item >= total) continue;
    const int y = (int)(item % a.h);
    const int stack = (int)((item / a.h) % 2);
    const int zl = (int)(item / (2L * a.h));
    const float* xr = (stack == 0 ? a.a : a.b) + ((size_t)(a.z0 + zl) * a.h + y) * a.w;
    auto load = [&](int n) -> float2 {
      const int x = 2 * n;
      return make_float2(x < a.w ? xr[x] : 0.f, x + 1 < a.w ? xr[x + 1] : 0.f);
    };
    auto sst = [&](int k, float2 v, int) { s[pad_idx(k)] = v; };
    team_fft<M, false>(s, tw, lane, team, load, sst);
    team_sync<C::LPV>(team);
    float2* dst = a.T + (size_t)item * a.NC;
    for (int k = lane; k <= M; k += C::LPV) {
      const float2 zk = s[pad_idx(k == M ? 0 : k)];
      const float2 zm = cconj(s[pad_idx(k == 0 ? 0 : M - k)]);
      const float2 e = cscale(cadd(zk, zm), 0.5f);
      const float2 d = csub(zk, zm);
      const float2 o = make_float2(0.5f * d.y, -0.5f * d.x);  // (zk - zm) / (2i)
      dst[k] = cadd(e, cmul(wq[k], o));
    }
  }
}

// ---------------------------------------------------------------------------
// columns: per NC-column tile, for each plane FFT_P(sample column) and
// FFT_P(PSF column), products accumulated per lane, added into St
// ---------------------------------------------------------------------------
template <int P>
struct ConvColCfg {
  using C0 = ColCfg<P>;
  static constexpr int LPV = C0::LPV;
  static constexpr bool CTA = C0::CTA;
  static constexpr int TW = tw_len(P);
  static constexpr size_t smem_for(int v) {
    return sizeof(float2) * ((size_t)TW + 2 * (size_t)v * col_len(P, v));
  }
  static constexpr int V0 = C0::V;
  static constexpr int V = smem_for(V0) <= 200 * 1024 ? V0 : (smem_for(V0 / 2) <= 200 * 1024 ? V0 / 2 : V0 / 4);
  static_assert(V >= 1 && (!CTA || (V * LPV) % 32 == 0), "convolution column tile");
  static constexpr int LEN = col_len(P, V);
  static constexpr int THREADS = V * LPV;
  static constexpr int MINB = 1;
  static constexpr size_t SMEM = smem_for(V);
  // rows >= h <= P / 2 are zero: the upper half of the first-stage inputs
  static constexpr unsigned ZM = [] {
    constexpr int R0 = Plan<P>::P.r[0];
    unsigned m = 0u;
    for (int r = R0 / 2; r < R0; ++r) m |= 1u << r;
    return R0 >= 2 ? m : 0u;
  }();
};

template <int P>
__global__ void __launch_bounds__(ConvColCfg<P>::THREADS, ConvColCfg<P>::MINB) k_conv_cols(ConvArgs a) {
  using Q = ConvColCfg<P>;
  constexpr int V = Q::V, LEN = Q::LEN, LPV = Q::LPV;
  constexpr int RL = Plan<P>::R_LAST, NBFL = P / RL, SLOTS = Plan<P>::OUT_SLOTS;
  static_assert(SLOTS == ((NBFL + LPV - 1) / LPV) * RL, "slot layout");
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* tA = sm + Q::TW;
  float2* tB = tA + V * LEN;
  load_twiddles<P>(tw, a.twg, threadIdx.x, blockDim.x);
  const int team = threadIdx.x / LPV, lane = threadIdx.x % LPV;
  float2* sA = tA + team * LEN;
  float2* sB = tB + team * LEN;
  const int tiles = (a.NC + V - 1) / V;
  for (int t = blockIdx.x; t < tiles; t += gridDim.x) {
    const int kc0 = t * V;
    float2 acc[SLOTS];
#pragma unroll
    for (int i = 0; i < SLOTS; ++i) acc[i] = make_float2(0.f, 0.f);
    for (int zl = 0; zl < a.zc; ++zl) {
      __syncthreads();
      const float2* TA = a.T + (size_t)(2 * zl) * a.h * a.NC;
      load_col_tile<V, LEN>(tA, TA, a.NC, kc0, a.NC, 0, a.h, [](int r) { return r; });
      load_col_tile<V, LEN>(tB, TA + (size_t)a.h * a.NC, a.NC, kc0, a.NC, 0, a.h, [](int r) { return r; });
      __syncthreads();
      auto ldA = [&](int n) -> float2 { return n < a.h ? sA[pad_idx(n)] : make_float2(0.f, 0.f); };
      auto stA = [&](int k, float2 v, int) { sA[pad_idx(k)] = v; };
      team_fft<P, false, LPV, Q::CTA, Q::ZM>(sA, tw, lane, team, ldA, stA);
      team_barrier<LPV, Q::CTA>(team);
      auto ldB = [&](int n) -> float2 { return n < a.h ? sB[pad_idx(n)] : make_float2(0.f, 0.f); };
      auto stAcc = [&](int k, float2 v, int slot) { acc[slot] = cadd(acc[slot], cmul(sA[pad_idx(k)], v)); };
      team_fft<P, false, LPV, Q::CTA, Q::ZM>(sB, tw, lane, team, ldB, stAcc);
    }
    // St[kc][k] += acc: the slot of output k = j + r NBF_last, j = lane + it LPV
    const int kc = kc0 + team;
    if (kc < a.NC) {
      float2* col = a.St + (size_t)kc * a.P;
#pragma unroll
      for (int slot = 0; slot < SLOTS; ++slot) {
        const int it = slot / RL, r = slot % RL;
        const int j = lane + it * LPV;
        if (j < NBFL) {
          const int k = j + r * NBFL;
          col[k] = cadd(col[k], acc[slot]);
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// final, columns: inverse FFT_P of each spectrum column (contiguous in St),
// only the crop rows written, transposed into U (NC, h)
// ---------------------------------------------------------------------------
template <int P>
__global__ void __launch_bounds__(RowCfg<P>::THREADS, RowCfg<P>::MINB) k_conv_fin_cols(ConvArgs a) {
  using C = RowCfg<P>;
  extern __shared__ float2 sm[];
  float2* tw = sm;
  load_twiddles<P>(tw, a.twg, threadIdx.x, blockDim.x);
  __syncthreads();
  const int team = threadIdx.x / C::LPV, lane = threadIdx.x % C::LPV;
  float2* s = sm + C::TW + team * Plan<P>::LEN;
  for (long base = (long)blockIdx.x * C::TEAMS; base < a.NC; base += (long)gridDim.x * C::TEAMS) {
    const long kc = base + team;
    if (kc >= a.NC) continue;
    const float2* src = a.St + (size_t)kc * a.P;
    float2* dst = a.U + (size_t)kc * a.h;
    auto load = [&](int n) -> float2 { return src[n]; };
    auto store = [&](int k, float2 v, int) {
      const int y = k - a.c0y;
      if (y >= 0 && y < a.h) dst[y] = v;
    };
    team_fft<P, true>(s, tw, lane, team, load, store);
  }
}

// ---------------------------------------------------------------------------
// final, rows: per output row (a column of U) the c2r of length Q through an
// inverse complex FFT of length M, the "same" crop and the scale
// ---------------------------------------------------------------------------
template <int M>
struct ConvFinCfg {
  using C0 = ColCfg<M>;
  static constexpr int LPV = C0::LPV;
  static constexpr bool CTA = C0::CTA;
  static constexpr int V = C0::V;
  static constexpr int LEN = col_len(2 * M, V);  // room for the M + 1 spectrum values
  static constexpr int TW = tw_len(M);
  static constexpr int THREADS = V * LPV;
  static constexpr int MINB = minb_for(THREADS);
  static constexpr size_t SMEM = sizeof(float2) * ((size_t)TW + (size_t)V * LEN);
};

template <int M>
__global__ void __launch_bounds__(ConvFinCfg<M>::THREADS, ConvFinCfg<M>::MINB) k_conv_fin_rows(ConvArgs a) {
  using Q = ConvFinCfg<M>;
  constexpr int V = Q::V, LEN = Q::LEN, LPV = Q::LPV;
  constexpr int QN = 2 * M;
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* tile = sm + Q::TW;
  load_twiddles<M>(tw, a.twg, threadIdx.x, blockDim.x);
  constexpr int OFF_Q = tw_offset(QN);
  const float2* wq = a.twg + OFF_Q;  // exp(-2 pi i k / Q)
  const int team = threadIdx.x / LPV, lane = threadIdx.x % LPV;
  float2* s = tile + team * LEN;
  const int tiles = (a.h + V - 1) / V;
  for (int t = blockIdx.x; t < tiles; t += gridDim.x) {
    const int y0 = t * V;
    __syncthreads();
    // Y[k] of output rows y0 .. y0 + V - 1: rows k < NC of U, columns y
    load_col_tile<V, LEN>(tile, a.U, a.h, y0, a.h, 0, a.NC, [](int r) { return r; });
    __syncthreads();
    // Z'[k] = E[k] + i O[k] in place, pairs (k, M - k) by one lane
    for (int k = lane; k <= M / 2; k += LPV) {
      const int km = M - k;
      const float2 yk = s[pad_idx(k)], ykm = s[pad_idx(km)];
      // k side
      {
        const float2 c = cconj(ykm);
        const float2 e = cscale(cadd(yk, c), 0.5f);
        const float2 w = cconj(wq[k]);  // W^-k
        const float2 o = cscale(cmul(csub(yk, c), w), 0.5f);
        s[pad_idx(k)] = make_float2(e.x - o.y, e.y + o.x);  // e + i o
      }
      if (km != k && km < M) {
        const float2 c = cconj(yk);
        const float2 e = cscale(cadd(ykm, c), 0.5f);
        const float2 w = cconj(wq[km]);
        const float2 o = cscale(cmul(csub(ykm, c), w), 0.5f);
        s[pad_idx(km)] = make_float2(e.x - o.y, e.y + o.x);
      }
    }
    team_barrier<LPV, Q::CTA>(team);
    const int y = y0 + team;
    float* orow = a.out + (size_t)(y < a.h ? y : 0) * a.w;
    const bool live = y < a.h;
    auto load = [&](int n) -> float2 { return s[pad_idx(n)]; };
    auto store = [&](int n, float2 v, int) {
      const int x0 = 2 * n - a.c0x, x1 = x0 + 1;
      if (live && x0 >= 0 && x0 < a.w) orow[x0] = v.x * a.scale;
      if (live && x1 >= 0 && x1 < a.w) orow[x1] = v.y * a.scale;
    };
    team_fft<M, true, LPV, Q::CTA>(s, tw, lane, team, load, store);
  }
}

cx_status conv_dispatch_rows(int m, const ConvArgs& a, cudaStream_t st);
cx_status conv_dispatch_cols(int p, const ConvArgs& a, cudaStream_t st);
cx_status conv_dispatch_fin_cols(int p, const ConvArgs& a, cudaStream_t st);
cx_status conv_dispatch_fin_rows(int m, const ConvArgs& a, cudaStream_t st);

}  // namespace cx
