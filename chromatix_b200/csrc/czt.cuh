// Chirp-Z transform along one axis (Bluestein), fused.
//
// Reference: utils/czt.py:7-52 (czt), 55-80 (cztn), 83-124 (zoomed_fft) and
// the CZT branch of kernel_propagate (functional/propagation.py:420-443).
//
// For each vector x (length n):
//   y[k] = w^(k^2/2) * sum_j x[j] a^(-j) w^(j^2/2) w^(-(k-j)^2/2),  k < m
// computed as a circular convolution of length L >= n + m - 1 (any compiled
// FFT length): the loader applies the input chirp (FP64 phase, reduced mod
// 2 pi), FFT_L, a multiply by the precomputed spectrum of the chirp filter,
// IFFT_L, and the store applies the output chirp, the optional modulation
// w^(-N k) a^N of the rescaled propagation and a real scale, writing only the
// m wanted outputs.
#pragma once

#include "host.cuh"

namespace cx {

struct CztArgs {
  int n, m, L;
  long n_vec;        // vectors v = o * inner + i
  int inner;
  long in_ostride, in_istride, in_estride;
  long out_ostride, out_istride, out_estride;
  double ta, tw;     // arg(a), arg(w)
  double la, lw;     // log|a|, log|w|
  int modN;          // >= 0: also multiply by w^(-modN k) a^modN
  double scale;      // real factor on the outputs
  const float2* chat;  // FFT_L of the chirp filter, 1/L folded in
  const float2* x;
  float2* y;
  const float2* twg;
  // kind 1: chirp convolution (the Yu et al. rescaling of kernel_propagate,
  // functional/propagation.py:445-458) instead of a chirp-Z transform:
  //   y[k] = mag_out exp(i pi c_out (dx_out (k - k0_out) + org_out)^2)
  //          * sum_j x[j] mag_in exp(i pi c_in (j - j0_in)^2) f[k + s - j],
  // with the finite chirp filter f in chat (see the filter kernel)
  int kind = 0;
  // kind 0: an extra output factor exp(k (gb_l + i gb_t) + c_l + i c_t) -- the
  // a-dependent part of the adjoint transform (zero for the forward one)
  double gb_l = 0.0, gb_t = 0.0, c_l = 0.0, c_t = 0.0;
  double c_in = 0.0, j0_in = 0.0, mag_in = 1.0;
  double c_out = 0.0, dx_out = 0.0, k0_out = 0.0, org_out = 0.0, mag_out = 1.0;
};

// a^(-j) w^(j^2/2)  (kind 1: the input factor of the chirp convolution)
__device__ __forceinline__ float2 czt_in_chirp(const CztArgs& a, int j) {
  if (a.kind == 1) {
    const double d = (double)j - a.j0_in;
    const float2 e = expi_reduced(3.141592653589793238462643383279502884 * a.c_in * d * d);
    return make_float2((float)a.mag_in * e.x, (float)a.mag_in * e.y);
  }
  const double jj = (double)j;
  const double lm = -a.la * jj + a.lw * 0.5 * jj * jj;
  const double ph = -a.ta * jj + a.tw * 0.5 * jj * jj;
  const float2 e = expi_reduced(ph);
  const float m = lm == 0.0 ? 1.f : (float)exp(lm);
  return make_float2(m * e.x, m * e.y);
}

// w^(k^2/2) [w^(-N k) a^N] * scale  (kind 1: the output factor of the chirp convolution)
__device__ __forceinline__ float2 czt_out_chirp(const CztArgs& a, int k) {
  if (a.kind == 1) {
    const double g = a.dx_out * ((double)k - a.k0_out) + a.org_out;
    const float2 e = expi_reduced(3.141592653589793238462643383279502884 * a.c_out * g * g);
    return make_float2((float)a.mag_out * e.x, (float)a.mag_out * e.y);
  }
  const double kk = (double)k;
  double lm = a.lw * 0.5 * kk * kk + a.gb_l * kk + a.c_l;
  double ph = a.tw * 0.5 * kk * kk + a.gb_t * kk + a.c_t;
  if (a.modN >= 0) {
    const double N = (double)a.modN;
    lm += -a.lw * N * kk + a.la * N;
    ph += -a.tw * N * kk + a.ta * N;
  }
  const float2 e = expi_reduced(ph);
  const float m = (float)(a.scale * (lm == 0.0 ? 1.0 : exp(lm)));
  return make_float2(m * e.x, m * e.y);
}

// vectors with contiguous or strided elements, one team per vector
template <int L>
__global__ void __launch_bounds__(RowCfg<L>::THREADS, RowCfg<L>::MINB) k_czt_rows(CztArgs a) {
  using C = RowCfg<L>;
  extern __shared__ float2 sm[];
  float2* tw = sm;
  load_twiddles<L>(tw, a.twg, threadIdx.x, blockDim.x);
  __syncthreads();
  const int team = threadIdx.x / C::LPV, lane = threadIdx.x % C::LPV;
  float2* s = sm + C::TW + team * Plan<L>::LEN;
  for (long base = (long)blockIdx.x * C::TEAMS; base < a.n_vec; base += (long)gridDim.x * C::TEAMS) {
    const long v = base + team;
    if (v >= a.n_vec) continue;
    const long o = v / a.inner, i = v % a.inner;
    const float2* xv = a.x + o * a.in_ostride + i * a.in_istride;
    float2* yv = a.y + o * a.out_ostride + i * a.out_istride;
    auto load = [&](int j) -> float2 {
      return j < a.n ? cmul(xv[(long)j * a.in_estride], czt_in_chirp(a, j)) : make_float2(0.f, 0.f);
    };
    auto st1 = [&](int k, float2 val, int) { s[pad_idx(k)] = cmul(val, a.chat[k]); };
    team_fft_ex<L, false, true, true>(s, tw, lane, team, load, st1);
    team_sync<C::LPV>(team);
    auto ld2 = [&](int k) -> float2 { return s[pad_idx(k)]; };
    auto st2 = [&](int k, float2 val, int) {
      const int r = k - (a.n - 1);
      if (r >= 0 && r < a.m) yv[(long)r * a.out_estride] = cmul(val, czt_out_chirp(a, r));
    };
    team_fft_ex<L, true, false, true>(s, tw, lane, team, ld2, st2);
  }
}

// vectors along a strided axis: V adjacent inner indices per CTA, tiles moved
// through shared memory with coalesced loads and stores
template <int L>
__global__ void __launch_bounds__(ColCfg<L>::THREADS, ColCfg<L>::MINB) k_czt_cols(CztArgs a) {
  using C = ColCfg<L>;
  constexpr int V = C::V, LEN = C::LEN;
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* tile = sm + C::TW;
  load_twiddles<L>(tw, a.twg, threadIdx.x, blockDim.x);
  const int team = threadIdx.x / C::LPV, lane = threadIdx.x % C::LPV;
  float2* s = tile + team * LEN;
  const int tiles_i = (a.inner + V - 1) / V;
  const long n_outer = a.n_vec / a.inner;
  const long total = (long)tiles_i * n_outer;
  for (long t = blockIdx.x; t < total; t += gridDim.x) {
    const long o = t / tiles_i;
    const int i0 = (int)(t % tiles_i) * V;
    __syncthreads();
    // tile rows j < n of vectors i0 .. i0 + V - 1 (in_istride == 1)
    load_col_tile<V, LEN>(tile, a.x + o * a.in_ostride, a.in_estride, i0, a.inner, 0, a.n, [](int r) { return r; });
    __syncthreads();
    auto load = [&](int j) -> float2 {
      return j < a.n ? cmul(s[pad_idx(j)], czt_in_chirp(a, j)) : make_float2(0.f, 0.f);
    };
    auto st1 = [&](int k, float2 val, int) { s[pad_idx(k)] = cmul(val, a.chat[k]); };
    team_fft_ex<L, false, true, true, C::LPV, C::CTA>(s, tw, lane, team, load, st1);
    team_barrier<C::LPV, C::CTA>(team);
    auto ld2 = [&](int k) -> float2 { return s[pad_idx(k)]; };
    auto st2 = [&](int k, float2 val, int) {
      const int r = k - (a.n - 1);
      if (r >= 0 && r < a.m) s[pad_idx(k)] = cmul(val, czt_out_chirp(a, r));
    };
    team_fft_ex<L, true, false, true, C::LPV, C::CTA>(s, tw, lane, team, ld2, st2);
    __syncthreads();
    float2* yo = a.y + o * a.out_ostride;
    for (int idx = threadIdx.x; idx < a.m * V; idx += blockDim.x) {
      const int r = idx / V, c = idx % V, i = i0 + c;
      if (i < a.inner) yo[(long)r * a.out_estride + i] = tile[c * LEN + pad_idx(a.n - 1 + r)];
    }
  }
}

cx_status czt_dispatch_rows(int L, const CztArgs& a, cudaStream_t st);
cx_status czt_dispatch_cols(int L, const CztArgs& a, cudaStream_t st);

}  // namespace cx
