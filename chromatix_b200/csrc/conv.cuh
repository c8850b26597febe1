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

// Transform lengths.  Any P >= h_a + h_b - 1 gives the same linear
// convolution after the "same" crop (the reference's next power of two
// included), so the column length P is the smallest even engine length
// >= 2 h and the row length Q = 2 M the smallest >= 2 w whose half M is an
// engine length; powers of two on request.
#define CX_CONV_P_SIZES(X)                                                                                   \
  X(2) X(4) X(6) X(8) X(10) X(12) X(14) X(16) X(20) X(24) X(28) X(32) X(40) X(48) X(56) X(64) X(80) X(96)    \
  X(112) X(128) X(160) X(192) X(224) X(256) X(320) X(384) X(448) X(512) X(640) X(768) X(896) X(1024) X(1280) \
  X(1536) X(1792) X(2048) X(2560) X(3072) X(3584) X(4096)
#define CX_CONV_M_SIZES(X)                                                                                  \
  X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(10) X(12) X(14) X(16) X(20) X(24) X(28) X(32) X(40) X(48) X(56) X(64) \
  X(80) X(96) X(112) X(128) X(160) X(192) X(224) X(256) X(320) X(384) X(448) X(512) X(640) X(768) X(896)    \
  X(1024) X(1280) X(1536) X(1792) X(2048)


struct ConvArgs {
  int h, w;               // image (sample) plane shape = output shape
  int kh, kw;             // kernel (PSF) plane shape
  int HB;                 // rows per tile block of T: max(h, kh)
  int NT, vt_shift;       // column tiles of T and their width VT = 1 << vt_shift (>= 4, a multiple of the column pass's V)
  int P, Q, M, NC;        // transform lengths, M = Q / 2, NC = M + 1
  int z0, zc;             // plane chunk
  const float* a;         // sample (n_planes, h, w)
  const float* b;         // kernel (n_planes, kh, kw), or one (kh, kw) plane
  long b_plane;           // kernel plane stride in floats (0: one kernel for all planes)
  float2* T;              // row spectra by column tile (zc, 2, NT, HB, VT): stack 0 rows < h, stack 1 rows < kh
  float2* St;             // accumulated spectrum, transposed (NC, P)
  float2* U;              // column inverse of the crop rows, transposed (NC, h)
  float* out;             // image (h, w)
  int c0y, c0x;           // "same" crop offsets ((kh - 1) / 2, (kw - 1) / 2)
  float scale;            // 2 / (P Q)
  const float2* twg;
};

// ---------------------------------------------------------------------------
// rows: r2c of the zc planes of both stacks (items: plane, stack, row).  T is
// stored by column tile, (zc, 2, NT, HB, VT) with VT = max(4, the column
// pass's tile width): a row's run in a tile is >= 32 bytes, so every lane
// group writes whole sectors (partial sectors make the L2 read them back
// from DRAM) and the column pass copies its columns from one block.
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
  static_assert(OFF_Q >= 0, "row length Q = 2 M has no twiddle table");
  const float2* wq = a.twg + OFF_Q;  // exp(-2 pi i k / Q), k < Q
  const int team = threadIdx.x / C::LPV, lane = threadIdx.x % C::LPV;
  float2* s = sm + C::TW + team * Plan<M>::LEN;
  const int vs = a.vt_shift, vm = (1 << a.vt_shift) - 1;
  const size_t tile_stride = (size_t)a.HB << vs;
  // items: (plane, stack, row), h sample rows then kh kernel rows per plane
  const int rows = a.h + a.kh;
  const long total = (long)a.zc * rows;
  for (long base = (long)blockIdx.x * C::TEAMS; base < total; base += (long)gridDim.x * C::TEAMS) {
    const long item = base + team;
    if (item >= total) continue;
    const int zl = (int)(item / rows), r = (int)(item % rows);
    const int stack = r < a.h ? 0 : 1;
    const int y = stack == 0 ? r : r - a.h;
    const int w = stack == 0 ? a.w : a.kw;
    const float* xr = stack == 0 ? a.a + ((size_t)(a.z0 + zl) * a.h + y) * a.w
                                 : a.b + (size_t)(a.z0 + zl) * a.b_plane + (size_t)y * a.kw;
    // even width on an 8-byte boundary: one float2 load per input pair
    const bool pairs = (w % 2) == 0 && (reinterpret_cast<uintptr_t>(xr) & 7u) == 0;
    auto load = [&](int n) -> float2 {
      const int x = 2 * n;
      if (pairs) return x < w ? __ldg(reinterpret_cast<const float2*>(xr + x)) : make_float2(0.f, 0.f);
      return make_float2(x < w ? xr[x] : 0.f, x + 1 < w ? xr[x + 1] : 0.f);
    };
    auto sst = [&](int k, float2 v, int) { s[pad_idx(k)] = v; };
    // z[n] = 0 for n >= ceil(w / 2), and Q >= 2 max(w, kw) puts that below M / 2
    team_fft<M, false, C::LPV, false, lower_half_mask<M>()>(s, tw, lane, team, load, sst);
    team_sync<C::LPV>(team);
    float2* dst = a.T + (size_t)(2 * zl + stack) * a.NT * tile_stride + ((size_t)y << vs);
    for (int k = lane; k <= M; k += C::LPV) {
      const float2 zk = s[pad_idx(k == M ? 0 : k)];
      const float2 zm = cconj(s[pad_idx(k == 0 ? 0 : M - k)]);
      const float2 e = cscale(cadd(zk, zm), 0.5f);
      const float2 d = csub(zk, zm);
      const float2 o = make_float2(0.5f * d.y, -0.5f * d.x);  // (zk - zm) / (2i)
      dst[(size_t)(k >> vs) * tile_stride + (k & vm)] = cadd(e, cmul(wq[k], o));
    }
  }
}

// ---------------------------------------------------------------------------
// columns: work units (column tile of V spectrum columns, plane), split in
// equal contiguous ranges over the CTAs (no last-wave tail).  Per unit:
// FFT_P of the sample column and of the PSF column, product accumulated per
// lane; the accumulators go to St (float2 atomicAdd) when the range leaves a
// tile.  The next unit's columns are copied into a staging area with
// cp.async while the current unit's transforms run (two copy groups, one
// per stack, double-buffered against the transforms):
//   wait A(u), FFT A(u), issue A(u+1) | wait B(u), FFT B(u) + acc, issue B(u+1)
// ---------------------------------------------------------------------------
template <int P>
struct ConvColCfg {
  using C0 = ColCfg<P>;
  static constexpr int LPV = C0::LPV;
  static constexpr bool CTA = C0::CTA;
  static constexpr int TW = tw_len(P);
  static constexpr int HS = P / 2;  // staging rows per column (h, kh <= P / 2)
  // twiddles | two transform tiles | staging [stack][column][HS]
  static constexpr int stg_off(int v) { return TW + 2 * v * col_len(P, v); }
  static constexpr size_t smem_for(int v) { return sizeof(float2) * ((size_t)stg_off(v) + 2 * (size_t)v * HS); }
  static constexpr int V0 = C0::V;
  // within 200 KB, and at most 384 threads so that the transform plus the
  // per-lane accumulators (about 150 registers at P >= 1024) fit without
  // spilling; exact-size teams keep whole warps
  static constexpr int pick_v() {
    int v = V0;
    while (v > 1 && smem_for(v) > 200 * 1024) v /= 2;
    while (v > 1 && v * LPV > 384 && (!CTA || ((v / 2) * LPV) % 32 == 0)) v /= 2;
    return v;
  }
  static constexpr int V = pick_v();
  static_assert(V >= 1 && (!CTA || (V * LPV) % 32 == 0), "convolution column tile");
  static constexpr int LEN = col_len(P, V);
  static constexpr int THREADS = V * LPV;
  static constexpr int MINB = 1;
  static constexpr size_t SMEM = smem_for(V);
  static_assert(SMEM <= 227 * 1024, "convolution column tile exceeds shared memory");
  // rows >= h (kh) are zero and P >= 2 max(h, kh)
  static constexpr unsigned ZM = lower_half_mask<P>();
};

template <int P>
__global__ void __launch_bounds__(ConvColCfg<P>::THREADS, ConvColCfg<P>::MINB) k_conv_cols(ConvArgs a) {
  using Q = ConvColCfg<P>;
  constexpr int V = Q::V, LEN = Q::LEN, LPV = Q::LPV, HS = Q::HS;
  // store slots of the last stage with this kernel's lane count:
  // slot = it R_last + r for output j + r NBF_last, j = lane + it LPV
  constexpr int RL = Plan<P>::R_LAST, NBFL = P / RL, SLOTS = ((NBFL + LPV - 1) / LPV) * RL;
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* tA = sm + Q::TW;
  float2* tB = tA + V * LEN;
  float2* stg = sm + Q::stg_off(V);  // [stack][V][HS]
  load_twiddles<P>(tw, a.twg, threadIdx.x, blockDim.x);
  const int team = threadIdx.x / LPV, lane = threadIdx.x % LPV;
  float2* sA = tA + team * LEN;
  float2* sB = tB + team * LEN;
  const float2* gA = stg + team * HS;
  const float2* gB = stg + (V + team) * HS;
  const long zc = a.zc;
  const long units = (long)((a.NC + V - 1) / V) * zc;
  const long u0 = units * blockIdx.x / gridDim.x, u1 = units * (blockIdx.x + 1) / gridDim.x;
  if (u0 >= u1) return;  // whole CTA, before any barrier
  // copy the stack's V columns of unit u (V of the VT columns of one T tile
  // block) into the staging area, one run per column; the columns past NC
  // of the last tile are never written by the row pass: their transforms
  // are computed and discarded
  const int vts = a.vt_shift;
  auto prefetch = [&](long u, int stack) {
    const int c0 = (int)(u / zc) * V, zl = (int)(u % zc);
    const float2* src = a.T + (((size_t)(2 * zl + stack) * a.NT + (c0 >> vts)) * a.HB << vts) +
                        (c0 & ((1 << vts) - 1));
    float2* dst = stg + stack * V * HS;
    const int n = (stack == 0 ? a.h : a.kh) * V;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const int y = i / V, c = i % V;
      cp_async8(dst + c * HS + y, src + ((size_t)y << vts) + c);
    }
  };
  float2 acc[SLOTS];
#pragma unroll
  for (int i = 0; i < SLOTS; ++i) acc[i] = make_float2(0.f, 0.f);
  prefetch(u0, 0);
  cp_async_commit();
  prefetch(u0, 1);
  cp_async_commit();
  for (long u = u0; u < u1; ++u) {
    const int t = (int)(u / zc);
    cp_async_wait_group<1>();  // A(u) (B(u) may be in flight)
    __syncthreads();
    auto ldA = [&](int n) -> float2 { return n < a.h ? gA[n] : make_float2(0.f, 0.f); };
    auto stA = [&](int k, float2 v, int) { sA[pad_idx(k)] = v; };
    team_fft<P, false, LPV, Q::CTA, Q::ZM>(sA, tw, lane, team, ldA, stA);
    __syncthreads();  // every team is past its reads of the A staging
    if (u + 1 < u1) prefetch(u + 1, 0);
    cp_async_commit();
    cp_async_wait_group<1>();  // B(u)
    __syncthreads();
    auto ldB = [&](int n) -> float2 { return n < a.kh ? gB[n] : make_float2(0.f, 0.f); };
    auto stAcc = [&](int k, float2 v, int slot) { acc[slot] = cadd(acc[slot], cmul(sA[pad_idx(k)], v)); };
    team_fft<P, false, LPV, Q::CTA, Q::ZM>(sB, tw, lane, team, ldB, stAcc);
    __syncthreads();  // B staging and the A tile are free
    if (u + 1 < u1) prefetch(u + 1, 1);
    cp_async_commit();
    if (u + 1 == u1 || (u + 1) / zc != t) {
      // St[kc][k] += acc for output k = j + r NBF_last of slot it R_last + r
      const int kc = t * V + team;
      if (kc < a.NC) {
        float2* col = a.St + (size_t)kc * a.P;
#pragma unroll
        for (int slot = 0; slot < SLOTS; ++slot) {
          const int it = slot / RL, r = slot % RL;
          const int j = lane + it * LPV;
          if (j < NBFL) atomicAdd(col + j + r * NBFL, acc[slot]);
        }
      }
#pragma unroll
      for (int i = 0; i < SLOTS; ++i) acc[i] = make_float2(0.f, 0.f);
    }
  }
  cp_async_wait_all();
}

// ---------------------------------------------------------------------------
// final, columns: inverse FFT_P of each spectrum column (contiguous in St),
// only the crop rows written, transposed into U (NC, h)
// ---------------------------------------------------------------------------
// no blocks-per-SM bound: the long transforms' unrolled stores need up to
// about 170 registers
template <int P>
__global__ void __launch_bounds__(RowCfg<P>::THREADS, 1) k_conv_fin_cols(ConvArgs a) {
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
  static_assert(SMEM <= 227 * 1024, "convolution row tile exceeds shared memory");
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
  static_assert(OFF_Q >= 0, "row length Q = 2 M has no twiddle table");
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
int conv_col_tile(int p);  // the column pass's tile width V for length p (0: unsupported)
cx_status conv_dispatch_cols(int p, const ConvArgs& a, cudaStream_t st);
cx_status conv_dispatch_fin_cols(int p, const ConvArgs& a, cudaStream_t st);
cx_status conv_dispatch_fin_rows(int m, const ConvArgs& a, cudaStream_t st);

}  // namespace cx
