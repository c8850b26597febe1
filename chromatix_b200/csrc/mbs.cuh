// Modified Born series: the preconditioned fixed-point iteration on a 3D grid.
//
// Reference: experimental/modified_born_series/solver.py:42-146 and
// sample.py:9-124.  With V(y) = y * (s eps - kb2) (shifted_discrepancy),
// G(y) = IFFT3[ Y_T / (kb2 - s |k|^2) + Y_L / kb2 ] (shifted_approx_inv,
// k normalised by k0, Y_L = k (k.Y)/|k|^2, Y_T = Y - Y_L) one iteration is
//   x <- prec_y - prec_forward(x) + x = prec_y + V(G(V x) + x) + x.
// The state is three component planes (X, Y, Z) complex64.  Passes:
//   Z  (lines along z)    load x, V x, FFT_z
//   Y  (column tiles)     FFT_y / IFFT_y in place
//   X  (column tiles, 3 components per CTA) FFT_x, k-space projection and
//      Green's-function division, IFFT_x
//   Zi (lines along z)    IFFT_z / (X Y Z) -> G; x_new = prec_y + V(G + x) + x,
//      FP64 partial sums of |x_new - x|^2 and |x_new|^2
#pragma once

#include "host.cuh"

namespace cx {

enum MbsZMode {
  MBS_Z_DISC = 0,   // buf = FFT_z(V x)                (forward operator input)
  MBS_Z_SCALE = 1,  // buf = FFT_z(s * src)            (preconditioned source)
  MBS_ZI_STEP = 2,  // x_new = prec_y + V(G + x) + x, residual sums
  MBS_ZI_PREC = 3   // prec_y = -V(G)
};

struct MbsArgs {
  int X, Y, Z;
  long vox;           // X * Y * Z
  float2 s, kb2;      // scale (1 / (1.1 i R)) and k_bias^2 = shift * scale + 1
  float kfx, kfy, kfz;  // 2 pi / (N spacing k0) per axis: k' = kf * fftfreq numerator
  const float2* eps;  // (X, Y, Z) permittivity
  const float2* x;    // current iterate (3 planes) / source for MBS_Z_SCALE
  const float2* prec_y;
  float2* buf;        // FFT work state (3 planes)
  float2* x_new;      // output (3 planes)
  double* acc;        // [0] sum |x_new - x|^2, [1] sum |x_new|^2
  const float2* twg;
  int forward_only = 0;  // MBS_ZI_STEP: write prec_forward(x) = -V(G + x) instead of the update (no sums)
};

__device__ __forceinline__ float2 mbs_disc(const MbsArgs& a, float2 v, float2 e) {
  // v * (s * eps - kb2)
  const float2 f = make_float2(a.s.x * e.x - a.s.y * e.y - a.kb2.x, a.s.x * e.y + a.s.y * e.x - a.kb2.y);
  return cmul(v, f);
}

// lines along z: one team per (ix, iy) line, the three components in turn,
// so the line's permittivity is read from HBM once (kept in shared memory)
template <int NZ, int MODE = MBS_Z_DISC>
struct MbsZCfg {
  using C = RowCfg<NZ>;
  // MBS_ZI_STEP: per team, the component's x and prec_y rows, copied in by
  // bulk (TMA) copies while the inverse transform runs, and their mbarrier
  static constexpr bool PREFETCH = MODE == MBS_ZI_STEP;
  static constexpr size_t PF_OFF = (C::SMEM + sizeof(float2) * (size_t)C::TEAMS * NZ + 15) & ~(size_t)15;
  static constexpr size_t BAR_OFF = PF_OFF + (PREFETCH ? sizeof(float2) * 2 * (size_t)C::TEAMS * NZ : 0);
  static constexpr size_t SMEM = BAR_OFF + (PREFETCH ? sizeof(uint64_t) * (size_t)C::TEAMS : 0);
  static constexpr int POLLS = 1 << 20;
};

template <int NZ, int MODE>
__global__ void __launch_bounds__(RowCfg<NZ>::THREADS, RowCfg<NZ>::MINB) k_mbs_z(MbsArgs a) {
  using C = RowCfg<NZ>;
  extern __shared__ float2 sm[];
  float2* tw = sm;
  load_twiddles<NZ>(tw, a.twg, threadIdx.x, blockDim.x);
  __syncthreads();
  const int team = threadIdx.x / C::LPV, lane = threadIdx.x % C::LPV;
  float2* s = sm + C::TW + team * Plan<NZ>::LEN;
  float2* se = sm + C::TW + C::TEAMS * Plan<NZ>::LEN + team * NZ;  // the line's permittivity
  using Q = MbsZCfg<NZ, MODE>;
  float2* pfx = reinterpret_cast<float2*>(reinterpret_cast<char*>(sm) + Q::PF_OFF) + (size_t)team * 2 * NZ;
  float2* pfp = pfx + NZ;
  uint64_t* bar = reinterpret_cast<uint64_t*>(reinterpret_cast<char*>(sm) + Q::BAR_OFF) + team;
  unsigned bphase = 0;
  // bulk copies need 16-byte aligned rows (even Z, aligned bases)
  const bool bulk_ok = Q::PREFETCH && (a.Z % 2 == 0) && ((reinterpret_cast<size_t>(a.x) & 15) == 0) &&
                       ((reinterpret_cast<size_t>(a.prec_y) & 15) == 0);
  if constexpr (Q::PREFETCH) {
    if (lane == 0) bulk_mbar_init(bar);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    __syncthreads();
  }
  const long lines = (long)a.X * a.Y;
  const float inv_n = 1.0f / ((float)a.X * (float)a.Y * (float)a.Z);
  double dsum = 0.0, nsum = 0.0;
  // L2 prefetch of the rows the team reads next (the next component of this
  // line, or the first of its next line with that line's permittivity),
  // issued while the current component is transformed
  const bool l2pf = (a.Z % 2 == 0) && ((reinterpret_cast<size_t>(a.x) & 15) == 0) &&
                    ((reinterpret_cast<size_t>(a.buf) & 15) == 0) &&
                    ((reinterpret_cast<size_t>(a.eps) & 15) == 0) &&
                    ((reinterpret_cast<size_t>(a.prec_y) & 15) == 0);
  auto prefetch_next = [&](long xy, int comp) {
    const long nxy = comp < 2 ? xy : xy + (long)gridDim.x * C::TEAMS;
    const int ncomp = comp < 2 ? comp + 1 : 0;
    if (!l2pf || lane != 0 || nxy >= lines) return;
    const unsigned rb = (unsigned)a.Z * 8u;
    const size_t noff = (size_t)ncomp * a.vox + (size_t)nxy * a.Z;
    if (ncomp == 0 && MODE != MBS_Z_SCALE) bulk_prefetch_l2(a.eps + (size_t)nxy * a.Z, rb);
    if constexpr (MODE == MBS_Z_DISC || MODE == MBS_Z_SCALE) {
      bulk_prefetch_l2(a.x + noff, rb);
    } else {
      bulk_prefetch_l2(a.buf + noff, rb);
      if constexpr (MODE == MBS_ZI_STEP) {
        bulk_prefetch_l2(a.x + noff, rb);
        bulk_prefetch_l2(a.prec_y + noff, rb);
      }
    }
  };
  for (long base = (long)blockIdx.x * C::TEAMS; base < lines; base += (long)gridDim.x * C::TEAMS) {
    const long xy = base + team;
    if (xy >= lines) continue;
    if constexpr (MODE != MBS_Z_SCALE) {
      const float2* erow = a.eps + (size_t)xy * a.Z;
      team_sync<C::LPV>(team);  // the previous line's reads of se are complete
      for (int k = lane; k < NZ; k += C::LPV) se[k] = erow[k];
      team_sync<C::LPV>(team);
    }
#pragma unroll 1
    for (int comp = 0; comp < 3; ++comp) {
      const size_t off = (size_t)comp * a.vox + (size_t)xy * a.Z;
      prefetch_next(xy, comp);
      float2* brow = a.buf + off;
      if constexpr (MODE == MBS_Z_DISC || MODE == MBS_Z_SCALE) {
        const float2* xrow = a.x + off;
        auto load = [&](int k) -> float2 {
          return MODE == MBS_Z_DISC ? mbs_disc(a, xrow[k], se[k]) : cmul(a.s, xrow[k]);
        };
        auto store = [&](int k, float2 v, int) { brow[k] = v; };
        team_fft_ex<NZ, false, true, false>(s, tw, lane, team, load, store);
      } else {
        auto load = [&](int k) -> float2 { return brow[k]; };
        if constexpr (MODE == MBS_ZI_STEP) {
          const float2* xrow = a.x + off;
          const float2* prow = a.prec_y + off;
          float2* orow = a.x_new + off;
          // the x and prec_y rows travel while the inverse transform runs; the
          // update then reads them from shared memory (or, if the bounded wait
          // ran out or the rows are not aligned, from global memory)
          team_sync<C::LPV>(team);  // the previous component's reads of the prefetch rows are complete
          if (bulk_ok && lane == 0) {
            const unsigned rb = (unsigned)a.Z * 8u;
            bulk_fence();
            bulk_expect(bar, 2u * rb);
            const uint64_t pol = l2_evict_first();
            bulk_copy_g2s_hint(pfx, xrow, rb, bar, pol);
            bulk_copy_g2s_hint(pfp, prow, rb, bar, pol);
          }
          auto keep = [&](int k, float2 g, int) { s[pad_idx(k)] = g; };
          team_fft_ex<NZ, true, false, false>(s, tw, lane, team, load, keep);
          bool pre = false;
          if (bulk_ok) {
            pre = bulk_wait(bar, bphase, Q::POLLS);
            bphase ^= 1u;
          }
          team_sync<C::LPV>(team);
#pragma unroll 2
          for (int k = lane; k < NZ; k += C::LPV) {
            const float2 xo = pre ? pfx[k] : xrow[k];
            const float2 gk = cscale(s[pad_idx(k)], inv_n);
            const float2 vx = mbs_disc(a, cadd(gk, xo), se[k]);
            if (a.forward_only) {
              orow[k] = make_float2(-vx.x, -vx.y);
              continue;
            }
            const float2 xn = cadd(cadd(pre ? pfp[k] : prow[k], vx), xo);
            orow[k] = xn;
            const float2 dd = csub(xn, xo);
            dsum += (double)dd.x * dd.x + (double)dd.y * dd.y;
            nsum += (double)xn.x * xn.x + (double)xn.y * xn.y;
          }
        } else {  // MBS_ZI_PREC: prec_y = -V(G)
          float2* orow = a.x_new + off;
          auto store = [&](int k, float2 g, int) {
            const float2 v = mbs_disc(a, cscale(g, inv_n), se[k]);
            orow[k] = make_float2(-v.x, -v.y);
          };
          team_fft_ex<NZ, true, false, true>(s, tw, lane, team, load, store);
        }
      }
    }
  }
  if constexpr (MODE == MBS_ZI_STEP) {
    // block reduction of the FP64 residual sums, one atomic pair per CTA
    __shared__ double red[2][32];
    for (int o = 16; o > 0; o >>= 1) {
      dsum += __shfl_xor_sync(0xffffffffu, dsum, o);
      nsum += __shfl_xor_sync(0xffffffffu, nsum, o);
    }
    const int wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    if ((threadIdx.x & 31) == 0) {
      red[0][wid] = dsum;
      red[1][wid] = nsum;
    }
    __syncthreads();
    if (threadIdx.x == 0 && a.acc) {
      double d0 = 0.0, n0 = 0.0;
      for (int w = 0; w < nw; ++w) {
        d0 += red[0][w];
        n0 += red[1][w];
      }
      atomicAdd(a.acc, d0);
      atomicAdd(a.acc + 1, n0);
    }
  }
}

// Asynchronous copy (cp.async, 8 bytes per element) of rows [0, n) x columns
// [x0, x0 + V) of a row-major matrix (leading dimension ld) into a column tile
// tile[c * LEN + pad_idx(r)]; columns at or beyond ncols are not copied (their
// entries are stale and their results are never stored).  The caller commits.
template <int V, int LEN>
__device__ __forceinline__ void prefetch_col_tile(float2* tile, const float2* src, long ld, long x0, long ncols,
                                                  int n) {
  for (int idx = threadIdx.x; idx < n * V; idx += blockDim.x) {
    const int r = idx / V, c = idx % V;
    if (x0 + c < ncols) cp_async8(tile + c * LEN + pad_idx(r), src + (long)r * ld + x0 + c);
  }
}

// column tiles along an axis of length N with element stride E: vectors
// (outer o, inner i), element j at buf + o * ostride + i + j * E; in place.
// Two tiles in shared memory: the copy of the CTA's next tile is in flight
// (cp.async) while the current one is transformed and stored.
// At least 8 columns per tile: each row of the strided axis is read and
// written as one 64-byte segment.
template <int N>
struct MbsColCfg {
  using B = ColCfg<N, false>;
  static constexpr int LPV = B::LPV, TW = B::TW;
  static constexpr bool CTA = B::CTA;
  static constexpr int V = B::V >= 8 ? B::V : (8 * LPV <= 1024 ? 8 : B::V);
  static constexpr int LEN = col_len(N, V);
  static constexpr int THREADS = V * LPV;
  static constexpr int MINB = minb_for(THREADS);
  static constexpr size_t SMEM = sizeof(float2) * ((size_t)TW + 2 * (size_t)V * LEN);
  static_assert(SMEM <= 227 * 1024, "two column tiles do not fit in shared memory");
  static_assert(!CTA, "column teams of the strided passes tile warps");
};

template <int N, bool INV>
__global__ void __launch_bounds__(MbsColCfg<N>::THREADS, MbsColCfg<N>::MINB) k_mbs_cols(MbsArgs a, long n_outer,
                                                                                int inner, long ostride, long E) {
  using C = MbsColCfg<N>;
  constexpr int V = C::V, LEN = C::LEN;
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* tiles = sm + C::TW;  // [2][V][LEN]
  load_twiddles<N>(tw, a.twg, threadIdx.x, blockDim.x);
  const int team = threadIdx.x / C::LPV, lane = threadIdx.x % C::LPV;
  const int tiles_i = (inner + V - 1) / V;
  const long total = (long)tiles_i * n_outer;
  auto prefetch = [&](long t, float2* tile) {
    const long o = t / tiles_i;
    prefetch_col_tile<V, LEN>(tile, a.buf + o * ostride, E, (t % tiles_i) * V, inner, N);
    cp_async_commit();
  };
  long t = blockIdx.x;
  if (t < total) prefetch(t, tiles);
  for (int b = 0; t < total; t += gridDim.x, b ^= 1) {
    float2* tile = tiles + b * V * LEN;
    const long o = t / tiles_i;
    const int i0 = (int)(t % tiles_i) * V;
    float2* base = a.buf + o * ostride;
    if (t + gridDim.x < total) {
      prefetch(t + gridDim.x, tiles + (b ^ 1) * V * LEN);
      cp_async_wait_group<1>();
    } else {
      cp_async_wait_group<0>();
    }
    __syncthreads();
    float2* s = tile + team * LEN;
    auto load = [&](int j) -> float2 { return s[pad_idx(j)]; };
    auto store = [&](int k, float2 v, int) { s[pad_idx(k)] = v; };
    team_fft<N, INV, C::LPV, C::CTA>(s, tw, lane, team, load, store);
    __syncthreads();
    for (int idx = threadIdx.x; idx < N * V; idx += blockDim.x) {
      const int r = idx / V, c = idx % V, i = i0 + c;
      if (i < inner) base[(long)r * E + i] = tile[c * LEN + pad_idx(r)];
    }
    __syncthreads();  // the next iteration's prefetch refills this tile
  }
}

// along x for all three components at once (inner = Y*Z, E = Y*Z), with the
// k-space projection / Green's-function division between FFT_x and IFFT_x
template <int NX>
struct MbsXCfg {
  using C = ColCfg<NX, false>;
  static constexpr int LPV = C::LPV;
  static constexpr bool CTA = C::CTA;
  // about 128 lanes per component (at least 4 columns), at most 1024 threads;
  // exact-size teams (CTA) fill whole warps
  static constexpr int V1 = LPV < 32 ? (pow2_floor(128 / LPV) > 4 ? pow2_floor(128 / LPV) : 4) : (3 * 8 * LPV <= 1024 ? 8 : 4);
  static constexpr int V0 = (CTA && (3 * V1 * LPV) % 32 != 0 && 3 * 2 * V1 * LPV <= 1024) ? 2 * V1 : V1;
  static constexpr int V = (3 * V0 * LPV <= 1024) ? V0 : ((3 * 2 * LPV <= 1024) ? 2 : 1);
  static_assert(!CTA || (3 * V * LPV) % 32 == 0, "exact-size teams must fill whole warps");
  static constexpr int LEN = col_len(NX, V);
  static constexpr int THREADS = 3 * V * LPV;
  static constexpr int MINB = minb_for(THREADS);
  // two tiles of three components: the next one is copied in (cp.async) while the current one is processed
  static constexpr size_t SMEM = sizeof(float2) * ((size_t)C::TW + 2 * 3 * (size_t)V * LEN);
  static_assert(SMEM <= 227 * 1024, "two x tiles do not fit in shared memory");
};

template <int NX>
__global__ void __launch_bounds__(MbsXCfg<NX>::THREADS, MbsXCfg<NX>::MINB) k_mbs_x(MbsArgs a) {
  using Q = MbsXCfg<NX>;
  constexpr int V = Q::V, LEN = Q::LEN, LPV = Q::LPV;
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* tiles_sm = sm + ColCfg<NX, false>::TW;  // [2][comp][V][LEN]
  load_twiddles<NX>(tw, a.twg, threadIdx.x, blockDim.x);
  const int team = threadIdx.x / LPV, lane = threadIdx.x % LPV;  // team = comp * V + column
  const long inner = (long)a.Y * a.Z;
  const long tiles = (inner + V - 1) / V;
  auto prefetch = [&](long t, float2* tile) {
    for (int c = 0; c < 3; ++c)
      prefetch_col_tile<V, LEN>(tile + c * V * LEN, a.buf + (size_t)c * a.vox, inner, t * V, inner, NX);
    cp_async_commit();
  };
  long t = blockIdx.x;
  if (t < tiles) prefetch(t, tiles_sm);
  for (int b = 0; t < tiles; t += gridDim.x, b ^= 1) {
    const long i0 = t * V;
    float2* tile = tiles_sm + b * 3 * V * LEN;
    float2* s = tile + team * LEN;
    if (t + gridDim.x < tiles) {
      prefetch(t + gridDim.x, tiles_sm + (b ^ 1) * 3 * V * LEN);
      cp_async_wait_group<1>();
    } else {
      cp_async_wait_group<0>();
    }
    __syncthreads();
    auto load = [&](int j) -> float2 { return s[pad_idx(j)]; };
    auto store = [&](int k, float2 v, int) { s[pad_idx(k)] = v; };
    team_fft<NX, false, LPV, Q::CTA>(s, tw, lane, team, load, store);
    __syncthreads();
    // k-space operator, cooperatively over (kx, column): blockDim.x is a
    // multiple of V, so each thread keeps one column c and its (ky, kz)
    {
      const int c = threadIdx.x % V;
      const long i = i0 + c;
      const bool col_ok = i < inner;
      const long ii = col_ok ? i : 0;
      const int iy = (int)(ii / a.Z), iz = (int)(ii - (long)iy * a.Z);
      const float kyv = a.kfy * (float)freq_index(iy, a.Y);
      const float kzv = a.kfz * (float)freq_index(iz, a.Z);
      const float kyz = kyv * kyv + kzv * kzv;
      // 1 / kb2 (longitudinal part), a per-call constant
      const float bn = a.kb2.x * a.kb2.x + a.kb2.y * a.kb2.y;
      const float2 il = make_float2(a.kb2.x / bn, -a.kb2.y / bn);
      for (int kx = threadIdx.x / V; col_ok && kx < NX; kx += blockDim.x / V) {
        const float kxv = a.kfx * (float)freq_index(kx, a.X);
        const float ksq = kxv * kxv + kyz;
        float2* p0 = tile + (0 * V + c) * LEN + pad_idx(kx);
        float2* p1 = tile + (1 * V + c) * LEN + pad_idx(kx);
        float2* p2 = tile + (2 * V + c) * LEN + pad_idx(kx);
        const float2 y0 = *p0, y1 = *p1, y2 = *p2;
        // longitudinal part k (k . y) / |k|^2 (zero at k = 0)
        float2 l0 = make_float2(0.f, 0.f), l1 = l0, l2 = l0;
        if (ksq != 0.f) {
          const float r = __frcp_rn(ksq);
          const float2 proj = make_float2((kxv * y0.x + kyv * y1.x + kzv * y2.x) * r,
                                          (kxv * y0.y + kyv * y1.y + kzv * y2.y) * r);
          l0 = cscale(proj, kxv);
          l1 = cscale(proj, kyv);
          l2 = cscale(proj, kzv);
        }
        // 1 / (kb2 - s ksq) = conj(dt) / |dt|^2
        const float2 dt = make_float2(a.kb2.x - a.s.x * ksq, a.kb2.y - a.s.y * ksq);
        const float rd = __frcp_rn(dt.x * dt.x + dt.y * dt.y);
        const float2 it = make_float2(dt.x * rd, -dt.y * rd);
        *p0 = cadd(cmul(csub(y0, l0), it), cmul(l0, il));
        *p1 = cadd(cmul(csub(y1, l1), it), cmul(l1, il));
        *p2 = cadd(cmul(csub(y2, l2), it), cmul(l2, il));
      }
    }
    __syncthreads();
    team_fft<NX, true, LPV, Q::CTA>(s, tw, lane, team, load, store);
    __syncthreads();
    for (int c = 0; c < 3; ++c) {
      float2* dst = a.buf + (size_t)c * a.vox;
      const float2* src = tile + c * V * LEN;
      for (int idx = threadIdx.x; idx < NX * V; idx += blockDim.x) {
        const int r = idx / V, cc = idx % V;
        const long i = i0 + cc;
        if (i < inner) dst[(long)r * inner + i] = src[cc * LEN + pad_idx(r)];
      }
    }
    __syncthreads();  // the next iteration's prefetch refills this tile
  }
}

cx_status mbs_dispatch_z(int n, int mode, const MbsArgs& a, cudaStream_t st);
cx_status mbs_dispatch_cols(int n, bool inv, const MbsArgs& a, long n_outer, int inner, long ostride, long E,
                            cudaStream_t st);
cx_status mbs_dispatch_x(int n, const MbsArgs& a, cudaStream_t st);

}  // namespace cx
