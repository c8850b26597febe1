// Column FFTs of length N = N1 * N2 on the tensor cores (four-step form,
// split FP16 precision), eight columns per CTA of 256 threads.
//
//   X[k1 + N1 k2] = sum_n2 W_N2^(n2 k2) W_N^(n2 k1) sum_n1 W_N1^(n1 k1) x[N2 n1 + n2]
//
// Stage 1: for every (n2, v) a length-N1 DFT over n1 -- one real GEMM per
// 128-row tile, rows m = n2 + N2 v, K = (re | im) of n1, the DFT matrix as B.
// Twiddle W_N^(n2 k1) in FP32 on the way out of tensor memory.
// Stage 2: for every (v, k1) a length-N2 DFT over n2 -- rows m = N1 v + k1.
// Both A operands are MN-major (rows contiguous within 16-byte chunks), so
// the loader writes eight consecutive input rows of one column as one chunk
// and a stage-1 thread (one row (n2, v)) writes its N1 outputs as N1/8 chunks
// of stage 2's A: no transposes through shared memory, and neighbouring lanes
// write neighbouring K columns (no bank conflicts).
//
// Precision: FP32 values enter as FP16 hi + lo pairs, D = Ahi Bhi + Alo Bhi +
// Ahi Blo in FP32 (tensor memory); the tile is scaled by a power of two
// (exact) per column so that column's largest input component is near 2^9,
// which keeps every stage-1 output below FP16's maximum (N1 * 2^9 sqrt 2 <
// 65504 for N1 <= 64) and puts hi and lo in FP16's normal range.  The
// relative error per transform is 2-5e-7 on the hardware (2-4x an FP32 FFT's;
// the split alone gives ~5e-8, the rest comes from the tensor core's FP32
// accumulation).
//
// The caller copies the prebuilt B1 / B2 (tc_fft_copy_b), allocates tensor memory
// (TMEM_COLS) and an mbarrier, and calls tc_fft_tile per column tile with a
// loader (column v of FFT rows n .. n+7) and a store (output bin k of column
// v).  Every mbarrier wait is bounded; tc_fft_tile returns false (uniformly
// over the CTA) if one ran out.
#pragma once
#include "host.cuh"
#include "tcgen05.cuh"

namespace cx {

template <int N1_, int N2_>
struct TcFft {
  static constexpr int N1 = N1_, N2 = N2_, N = N1 * N2;
  static constexpr int V = 8, THREADS = 256;
  static constexpr int M1 = V * N2, T1 = M1 / 128;          // stage-1 rows (n2, v), tiles
  static constexpr int M2 = V * N1, T2 = (M2 + 127) / 128;  // stage-2 rows (v, k1), tiles (last one padded)
  static constexpr int K1 = 2 * N1, K2 = 2 * N2;           // (re | im) inputs = outputs per stage
  static constexpr uint32_t A1_TILE = 128u * K1 * 2u;       // bytes of one tile of hi (or lo)
  static constexpr uint32_t A2_TILE = 128u * K2 * 2u;
  static constexpr uint32_t A1_BYTES = 2u * T1 * A1_TILE;   // hi tiles, then lo tiles
  static constexpr uint32_t A2_BYTES = 2u * T2 * A2_TILE;
  static constexpr uint32_t A_BYTES = A1_BYTES > A2_BYTES ? A1_BYTES : A2_BYTES;  // stage 2 reuses stage 1's space
  static constexpr uint32_t B1_BYTES = 2u * K1 * K1 * 2u;   // hi, lo
  static constexpr uint32_t B2_BYTES = 2u * K2 * K2 * 2u;
  static constexpr uint32_t SMEM = A_BYTES + B1_BYTES + B2_BYTES;
  static constexpr int RPT = N / THREADS;                   // input rows per thread
  static constexpr int TMEM_NEED = (T1 * K1 > T2 * K2) ? T1 * K1 : T2 * K2;
  static constexpr int TMEM_COLS = TMEM_NEED <= 64 ? 64 : TMEM_NEED <= 128 ? 128 : TMEM_NEED <= 256 ? 256 : 512;
  static constexpr int POLLS = 1 << 18;
  static_assert(N1 % 8 == 0 && N2 % 16 == 0 && M1 % 128 == 0, "tile shapes");
  static_assert(T1 == 2, "one stage-1 row per thread (256 threads, two 128-row tiles)");
  static_assert(K1 <= 256 && K2 <= 256 && K1 % 16 == 0 && K2 % 16 == 0, "MMA N / K");
  static_assert(N % THREADS == 0, "rows per thread");
  static_assert(N1 <= 64, "stage-1 output range stays inside FP16");
};

// device addresses of a transform's two DFT matrices (tc_dft_mats)
struct TcMats {
  const uint8_t* b1;
  const uint8_t* b2;
  int* timeouts;  // bumped once per CTA whose MMA wait ran out (cx_tc_timeouts)
};
inline cx_status tc_mats(int n1, int n2, TcMats* m) {
  m->b1 = tc_dft_mats(n1);
  m->b2 = tc_dft_mats(n2);
  m->timeouts = tc_timeout_counter();
  if (!m->b1 || !m->b2 || !m->timeouts) {
    set_error("tensor-core DFT matrices of lengths %d / %d are not on the device (cx_init)", n1, n2);
    return CX_ERR_CUDA;
  }
  return CX_OK;
}

struct TcFftSmem {
  uint8_t* A;   // A1 / A2 (hi tiles then lo tiles)
  uint8_t* B1;  // hi then lo
  uint8_t* B2;
  uint64_t* bar;
  float* red;   // 64 floats: per-warp column maxima (kept until the tile's output is stored)
};

// real-expanded DFT matrix of length R as a K-major B operand (2R x 2R):
// row j = output (re | im), column k = input (re | im); hi at B, lo at B + 4 R^2 bytes
template <int R>
__device__ void tc_fft_build_b(uint8_t* B, bool inverse, int tid, int nthreads) {
  constexpr int K = 2 * R;
  const double sgn = inverse ? 1.0 : -1.0;
  for (int idx = tid; idx < K * K; idx += nthreads) {
    const int j = idx / K, k = idx % K;
    const int n = k % R, kk = j % R, pin = k / R, pout = j / R;
    double sd, cd;
    sincospi(sgn * 2.0 * (double)((n * kk) % R) / (double)R, &sd, &cd);
    const float v = (float)(pin == pout ? cd : (pin == 0 ? sd : -sd));
    const __half h = __float2half_rn(v);
    const __half l = __float2half_rn(v - __half2float(h));
    *reinterpret_cast<__half*>(B + tc::off_kmajor(K, j, k)) = h;
    *reinterpret_cast<__half*>(B + K * K * 2 + tc::off_kmajor(K, j, k)) = l;
  }
}

// a CTA gave up on an MMA wait: count it once for the host (cx_tc_timeouts)
__device__ __forceinline__ void tc_note_timeout(const TcMats& m) {
  if (threadIdx.x == 0) atomicAdd(m.timeouts, 1);
}

// copy the prebuilt DFT matrices (tc_dft_mats: hi then lo, `bytes` in all)
// into shared memory, 16 bytes per thread and step
__device__ __forceinline__ void tc_fft_copy_b(uint8_t* dst, const uint8_t* __restrict__ src, uint32_t bytes, int tid,
                                              int nthreads) {
  const uint4* s4 = reinterpret_cast<const uint4*>(src);
  uint4* d4 = reinterpret_cast<uint4*>(dst);
  for (uint32_t i = tid; i < bytes / 16; i += nthreads) d4[i] = s4[i];
}

// 8 values (one 16-byte chunk of an operand) split and stored as hi / lo
__device__ __forceinline__ void tc_store_chunk(uint8_t* hi_base, uint8_t* lo_base, uint32_t off, const float* v8) {
  uint32_t hi[4], lo[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) tc::split2(v8[2 * q], v8[2 * q + 1], hi[q], lo[q]);
  *reinterpret_cast<uint4*>(hi_base + off) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
  *reinterpret_cast<uint4*>(lo_base + off) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
}

// Column-tile input phase shared by tc_fft_tile and tc_fft_mult_tile.
// Stage-1 rows are m = n2 + N2 v (column-major by tile column v), so an
// MN-major 16-byte chunk is eight consecutive input rows n = N2 n1 + n2 of one
// column.  Chunk q = tid + 256 i is (n1, v, n2 group g): lanes take n1 % 8
// fastest, then v % 4, so one load instruction reads 32 contiguous bytes of
// eight rows and the eight lanes of a store phase write eight consecutive K
// columns (16 bytes apart: no bank conflicts).  load8(n, v, out[8]): column v
// of input rows n .. n+7.  Each column is scaled by a power of two that puts
// its largest component near 2^9; the per-warp column maxima stay in S.red.
template <class F>
__device__ __forceinline__ void tc_col_chunk(int q, int& n1, int& v, int& g) {
  const int rest = q >> 5, r2 = rest >> 1;
  n1 = (r2 % (F::N1 / 8)) * 8 + (q & 7);
  g = r2 / (F::N1 / 8);
  v = (rest & 1) * 4 + ((q >> 3) & 3);
}

__device__ __forceinline__ float tc_scale_of(const float* red, int v) {
  float m = red[v];
#pragma unroll
  for (int w = 1; w < 8; ++w) m = fmaxf(m, red[w * 8 + v]);
  int e = 0;
  if (m > 0.f) frexpf(m, &e);
  return ldexpf(1.f, 9 - e);
}

template <class F, class Load8>
__device__ __forceinline__ void tc_col_input(const TcFftSmem& S, Load8 load8) {
  constexpr int N1 = F::N1, N2 = F::N2;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  float2 xv[F::RPT][8];
  float mx[8];
#pragma unroll
  for (int v = 0; v < 8; ++v) mx[v] = 0.f;
#pragma unroll
  for (int i = 0; i < F::RPT; ++i) {
    int n1, v, g;
    tc_col_chunk<F>(tid + i * F::THREADS, n1, v, g);
    load8(N2 * n1 + 8 * g, v, xv[i]);
    float m = 0.f;
#pragma unroll
    for (int j = 0; j < 8; ++j) m = fmaxf(m, fmaxf(fabsf(xv[i][j].x), fabsf(xv[i][j].y)));
#pragma unroll
    for (int r = 0; r < 8; ++r) mx[r] = (r == v) ? fmaxf(mx[r], m) : mx[r];
  }
#pragma unroll
  for (int v = 0; v < 8; ++v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx[v] = fmaxf(mx[v], __shfl_xor_sync(0xffffffffu, mx[v], o));
  }
  if (lane == 0) {
#pragma unroll
    for (int v = 0; v < 8; ++v) S.red[warp * 8 + v] = mx[v];
  }
  __syncthreads();
  uint8_t* Ahi = S.A;
  uint8_t* Alo = S.A + F::T1 * F::A1_TILE;
#pragma unroll
  for (int i = 0; i < F::RPT; ++i) {
    int n1, v, g;
    tc_col_chunk<F>(tid + i * F::THREADS, n1, v, g);
    const float s = tc_scale_of(S.red, v);
    float re[8], im[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      re[j] = xv[i][j].x * s;
      im[j] = xv[i][j].y * s;
    }
    const int m0 = 8 * g + N2 * v;
    const uint32_t tile = (uint32_t)(m0 >> 7) * F::A1_TILE;
    tc_store_chunk(Ahi + tile, Alo + tile, tc::off_mnmajor(128, m0 & 127, n1), re);
    tc_store_chunk(Ahi + tile, Alo + tile, tc::off_mnmajor(128, m0 & 127, N1 + n1), im);
  }
}

// Issue D[t] = A[t] B for T row tiles of 128 (3 split products per K step of
// 16) and commit them to the mbarrier; called by one thread.  A tiles of
// `tile_bytes` (hi tiles then lo tiles from `a`), B (K x K, K-major, hi then
// lo), D[t] at tensor-memory columns tmem + t K.
template <int K, int T>
__device__ __forceinline__ void tc_issue(uint64_t* bar, uint32_t tmem, const uint8_t* a, uint32_t tile_bytes,
                                         int a_mn, const uint8_t* b) {
  tc::fence_after_sync();
  const uint32_t id = tc::idesc_f16_f32(128, K, a_mn, 0);
  constexpr uint32_t a_lbo = 16 * 128, b_lbo = (K / 8) * 128;
  const uint32_t bh = tc::smem_u32(b), bl = bh + K * K * 2;
  const uint32_t a0 = tc::smem_u32(a), lo_off = T * tile_bytes;
#pragma unroll
  for (int t = 0; t < T; ++t) {
    const uint32_t ah = a0 + t * tile_bytes, al = ah + lo_off;
#pragma unroll
    for (int s = 0; s < K / 16; ++s) {
      const uint64_t dah = tc::smem_desc(ah + s * 2 * a_lbo, a_lbo, 128);
      const uint64_t dal = tc::smem_desc(al + s * 2 * a_lbo, a_lbo, 128);
      const uint64_t dbh = tc::smem_desc(bh + s * 2 * b_lbo, b_lbo, 128);
      const uint64_t dbl = tc::smem_desc(bl + s * 2 * b_lbo, b_lbo, 128);
      tc::mma_f16(tmem + t * K, dah, dbh, id, s > 0 ? 1u : 0u);
      tc::mma_f16(tmem + t * K, dal, dbh, id, 1u);
      tc::mma_f16(tmem + t * K, dah, dbl, id, 1u);
    }
  }
  tc::mma_commit(bar);
}

// the operand writes of this CTA are complete and visible to the tensor
// core; thread 0 then issues the GEMM and everyone waits for it (bounded)
template <int K, int T>
__device__ __forceinline__ bool tc_gemm(const TcFftSmem& S, uint32_t tmem, uint32_t& phase, const uint8_t* a,
                                        uint32_t tile_bytes, int a_mn, const uint8_t* b, int polls) {
  tc::fence_smem_to_async();
  tc::fence_before_sync();
  __syncthreads();
  if (threadIdx.x == 0) tc_issue<K, T>(S.bar, tmem, a, tile_bytes, a_mn, b);
  const bool ok = tc::mbar_wait(S.bar, phase, polls);
  phase ^= 1u;
  if (!__syncthreads_and(ok)) return false;
  tc::fence_after_sync();
  return true;
}

// One tile of eight columns.  load8(n, v, float2 out[8]): column v of FFT
// input rows n .. n+7 (tc_col_input); store(k, v, X): output bin k of column v.  tw: twiddles
// exp(-2 pi i e / N), e < N (shared or global).  Returns false if an MMA wait
// ran out (then no output was stored for this tile).
template <class F, class Load8, class Store>
__device__ bool tc_fft_tile(const TcFftSmem& S, uint32_t tmem, uint32_t& phase, const float2* __restrict__ tw,
                            bool inverse, Load8 load8, Store store) {
  constexpr int N1 = F::N1, N2 = F::N2, N = F::N, K1 = F::K1, K2 = F::K2;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  // ---- load, per-column power-of-two scale, stage-1 A (MN-major): row
  // m = n2 + N2 v, column k = part N1 + n1
  tc_col_input<F>(S, load8);
  uint8_t* A1hi = S.A;
  uint8_t* A1lo = S.A + F::T1 * F::A1_TILE;
  tc::fence_smem_to_async();
  tc::fence_before_sync();
  __syncthreads();
  if (tid == 0) {
    tc::fence_after_sync();
    constexpr uint32_t id1 = tc::idesc_f16_f32(128, K1, 1, 0);
    constexpr uint32_t a_lbo = 16 * 128, b_lbo = (K1 / 8) * 128;
    const uint32_t b1h = tc::smem_u32(S.B1), b1l = b1h + K1 * K1 * 2;
#pragma unroll
    for (int t = 0; t < F::T1; ++t) {
      const uint32_t ah = tc::smem_u32(A1hi) + t * F::A1_TILE, al = tc::smem_u32(A1lo) + t * F::A1_TILE;
      const uint32_t d = tmem + t * K1;
#pragma unroll
      for (int s = 0; s < K1 / 16; ++s) {
        const uint64_t dah = tc::smem_desc(ah + s * 2 * a_lbo, a_lbo, 128);
        const uint64_t dal = tc::smem_desc(al + s * 2 * a_lbo, a_lbo, 128);
        const uint64_t dbh = tc::smem_desc(b1h + s * 2 * b_lbo, b_lbo, 128);
        const uint64_t dbl = tc::smem_desc(b1l + s * 2 * b_lbo, b_lbo, 128);
        tc::mma_f16(d, dah, dbh, id1, s > 0 ? 1u : 0u);
        tc::mma_f16(d, dal, dbh, id1, 1u);
        tc::mma_f16(d, dah, dbl, id1, 1u);
      }
    }
    tc::mma_commit(S.bar);
  }
  bool ok = tc::mbar_wait(S.bar, phase, F::POLLS);
  phase ^= 1u;
  if (!__syncthreads_and(ok)) return false;
  tc::fence_after_sync();

  // ---- stage-1 result: thread = row (n2, v) of tile warp / 4; twiddle; stage-2 A
  {
    const int t = warp >> 2;
    const int m = t * 128 + (warp & 3) * 32 + lane;
    const int n2 = m % N2, v = m / N2;  // stage-1 row m = n2 + N2 v
    float d[K1];
#pragma unroll
    for (int c = 0; c < K1; c += 16) tc::tmem_ld16(tmem + ((uint32_t)((warp & 3) * 32) << 16) + t * K1 + c, d + c);
    tc::tmem_wait_ld();
    uint8_t* A2hi = S.A;
    uint8_t* A2lo = S.A + F::T2 * F::A2_TILE;
#pragma unroll
    for (int c = 0; c < N1 / 8; ++c) {
      float re[8], im[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int k1 = 8 * c + q;
        int ex = n2 * k1;
        ex = ex - (ex / N) * N;
        const float2 w = tw[ex];
        const float wr = w.x, wi = inverse ? -w.y : w.y;
        const float a = d[k1], b = d[N1 + k1];
        re[q] = a * wr - b * wi;
        im[q] = a * wi + b * wr;
      }
      const int m2 = v * N1 + 8 * c;  // 8 consecutive rows (v, k1)
      const uint32_t tile = (uint32_t)(m2 >> 7) * F::A2_TILE;
      tc_store_chunk(A2hi + tile, A2lo + tile, tc::off_mnmajor(128, m2 & 127, n2), re);
      tc_store_chunk(A2hi + tile, A2lo + tile, tc::off_mnmajor(128, m2 & 127, N2 + n2), im);
    }
  }
  tc::fence_smem_to_async();
  tc::fence_before_sync();
  __syncthreads();
  if (tid == 0) {
    tc::fence_after_sync();
    constexpr uint32_t id2 = tc::idesc_f16_f32(128, K2, 1, 0);
    constexpr uint32_t a_lbo = 16 * 128, b_lbo = (K2 / 8) * 128;
    uint8_t* A2hi = S.A;
    uint8_t* A2lo = S.A + F::T2 * F::A2_TILE;
    const uint32_t b2h = tc::smem_u32(S.B2), b2l = b2h + K2 * K2 * 2;
#pragma unroll
    for (int j = 0; j < F::T2; ++j) {
      const uint32_t ah = tc::smem_u32(A2hi) + j * F::A2_TILE, al = tc::smem_u32(A2lo) + j * F::A2_TILE;
      const uint32_t d = tmem + j * K2;
#pragma unroll
      for (int s = 0; s < K2 / 16; ++s) {
        const uint64_t dah = tc::smem_desc(ah + s * 2 * a_lbo, a_lbo, 128);
        const uint64_t dal = tc::smem_desc(al + s * 2 * a_lbo, a_lbo, 128);
        const uint64_t dbh = tc::smem_desc(b2h + s * 2 * b_lbo, b_lbo, 128);
        const uint64_t dbl = tc::smem_desc(b2l + s * 2 * b_lbo, b_lbo, 128);
        tc::mma_f16(d, dah, dbh, id2, s > 0 ? 1u : 0u);
        tc::mma_f16(d, dal, dbh, id2, 1u);
        tc::mma_f16(d, dah, dbl, id2, 1u);
      }
    }
    tc::mma_commit(S.bar);
  }
  ok = tc::mbar_wait(S.bar, phase, F::POLLS);
  phase ^= 1u;
  if (!__syncthreads_and(ok)) return false;
  tc::fence_after_sync();

  // ---- stage-2 result: row (v, k1) holds X[k1 + N1 k2], k2 < N2
#pragma unroll
  for (int j0 = 0; j0 < F::T2; j0 += 2) {
    const int j = j0 + (warp >> 2);
    if (j < F::T2) {  // whole warps: tcgen05.ld is warp-collective
      float d[K2];
#pragma unroll
      for (int c = 0; c < K2; c += 16) tc::tmem_ld16(tmem + ((uint32_t)((warp & 3) * 32) << 16) + j * K2 + c, d + c);
      tc::tmem_wait_ld();
      const int m2 = j * 128 + (warp & 3) * 32 + lane;
      if (m2 < F::M2) {
        const int v = m2 / N1, k1 = m2 - v * N1;
        float mv = S.red[v];
#pragma unroll
        for (int w = 1; w < 8; ++w) mv = fmaxf(mv, S.red[w * 8 + v]);
        int e = 0;
        if (mv > 0.f) frexpf(mv, &e);
        const float isc = ldexpf(1.f, e - 9);
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) store(k1 + N1 * k2, v, make_float2(d[k2] * isc, d[N2 + k2] * isc));
      }
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  return true;
}

// Fourier multiplier on eight columns: X = FFT_N(x) (forward four-step as in
// tc_fft_tile), Y = mult(k, v, X) (e.g. X H(k, kx)), then the unnormalised
// inverse transform in the transposed order, which starts from the rows
// (v, k1) that the forward pass leaves in tensor memory:
//   y[n2 + N2 n1] = sum_k1 W_N1^(-n1 k1) W_N^(-n2 k1) sum_k2 W_N2^(-n2 k2) Y[k1 + N1 k2],
// with IDFT(u) = conj(DFT(conj(u))) so both inverse stages reuse B1 and B2.
// Y is scaled by 2^-ceil(log2 N) before the inverse stages (|Y| <= N max|x|
// for |H| <= 1); the result handed to store_rows is exact up to rounding:
// y = N * IFFT(Y) (unnormalised).  store_row(n, const float2 row[8]) writes
// output row n (8 columns); the rows are staged in shared memory first.
template <class F, class Load8, class Mult, class StoreRow>
__device__ bool tc_fft_mult_tile(const TcFftSmem& S, uint32_t tmem, uint32_t& phase, const float2* __restrict__ tw,
                                 Load8 load8, Mult mult, StoreRow store_row) {
  constexpr int N1 = F::N1, N2 = F::N2, N = F::N, K1 = F::K1, K2 = F::K2;
  constexpr int LOG2N = N <= 1024 ? 10 : (N <= 2048 ? 11 : 12);
  constexpr int ROUNDS = (F::T2 + 1) / 2;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t wl = (uint32_t)((warp & 3) * 32) << 16;

  // ---- forward stages (as tc_fft_tile)
  tc_col_input<F>(S, load8);
  uint8_t* Ahi = S.A;
  if (!tc_gemm<K1, F::T1>(S, tmem, phase, S.A, F::A1_TILE, 1, S.B1, F::POLLS)) return false;
  {
    const int t = warp >> 2;
    const int m = t * 128 + (warp & 3) * 32 + lane;
    const int n2 = m % N2, v = m / N2;  // stage-1 row m = n2 + N2 v
    float d[K1];
#pragma unroll
    for (int c = 0; c < K1; c += 16) tc::tmem_ld16(tmem + wl + t * K1 + c, d + c);
    tc::tmem_wait_ld();
#pragma unroll
    for (int c = 0; c < N1 / 8; ++c) {
      float re[8], im[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int k1 = 8 * c + q;
        const float2 w = tw[(n2 * k1) % N];
        re[q] = d[k1] * w.x - d[N1 + k1] * w.y;
        im[q] = d[k1] * w.y + d[N1 + k1] * w.x;
      }
      const int m2 = v * N1 + 8 * c;
      const uint32_t tile = (uint32_t)(m2 >> 7) * F::A2_TILE;
      tc_store_chunk(Ahi + tile, Ahi + F::T2 * F::A2_TILE + tile, tc::off_mnmajor(128, m2 & 127, n2), re);
      tc_store_chunk(Ahi + tile, Ahi + F::T2 * F::A2_TILE + tile, tc::off_mnmajor(128, m2 & 127, N2 + n2), im);
    }
  }
  if (!tc_gemm<K2, F::T2>(S, tmem, phase, S.A, F::A2_TILE, 1, S.B2, F::POLLS)) return false;

  // ---- multiplier on the rows (v, k1) (each holds every k2); the inverse
  // stage A operand (K-major: row (v, k1), column (re | im) of k2) is written
  // row by row into the space of stage 2's operand, whose GEMM has completed
  // (tensor memory is overwritten only after the next barrier)
  const float rs = ldexpf(1.f, -LOG2N);
#pragma unroll
  for (int r = 0; r < ROUNDS; ++r) {
    const int j = 2 * r + (warp >> 2);
    if (j < F::T2) {
      float y[K2];
#pragma unroll
      for (int c = 0; c < K2; c += 16) tc::tmem_ld16(tmem + wl + j * K2 + c, y + c);
      tc::tmem_wait_ld();
      const int rl = (warp & 3) * 32 + lane;
      const int m2 = j * 128 + rl;
      if (m2 < F::M2) {
        const int v = m2 / N1, k1 = m2 - v * N1;
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) {
          const float2 Y = mult(k1 + N1 * k2, v, make_float2(y[k2], y[N2 + k2]));
          y[k2] = Y.x * rs;
          y[N2 + k2] = -Y.y * rs;  // conj: the inverse stage runs the forward DFT matrix
        }
      } else {
#pragma unroll
        for (int c = 0; c < K2; ++c) y[c] = 0.f;  // padding rows of the last tile
      }
      const uint32_t tile = (uint32_t)j * F::A2_TILE;
#pragma unroll
      for (int c = 0; c < K2 / 8; ++c)
        tc_store_chunk(Ahi + tile, Ahi + F::T2 * F::A2_TILE + tile, tc::off_kmajor(128, rl, 8 * c), y + 8 * c);
    }
  }
  if (!tc_gemm<K2, F::T2>(S, tmem, phase, S.A, F::A2_TILE, 0, S.B2, F::POLLS)) return false;

  // ---- D_A row (v, k1) = DFT_N2(conj Y) over k2 -> n2; times W_N^(n2 k1);
  // inverse stage B operand, MN-major: row (v, n2) = N2 v + n2, column (re | im) of k1
#pragma unroll
  for (int r = 0; r < ROUNDS; ++r) {
    const int j = 2 * r + (warp >> 2);
    if (j < F::T2) {
      float d[K2];
#pragma unroll
      for (int c = 0; c < K2; c += 16) tc::tmem_ld16(tmem + wl + j * K2 + c, d + c);
      tc::tmem_wait_ld();
      const int m2 = j * 128 + (warp & 3) * 32 + lane;
      if (m2 < F::M2) {
        const int v = m2 / N1, k1 = m2 - v * N1;
#pragma unroll
        for (int c = 0; c < N2 / 8; ++c) {
          float re[8], im[8];
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            const int n2 = 8 * c + q;
            const float2 w = tw[(n2 * k1) % N];
            re[q] = d[n2] * w.x - d[N2 + n2] * w.y;
            im[q] = d[n2] * w.y + d[N2 + n2] * w.x;
          }
          const int mb = v * N2 + 8 * c;
          const uint32_t tile = (uint32_t)(mb >> 7) * F::A1_TILE;
          // stage A's operand (K-major) is no longer read: the GEMM has completed
          tc_store_chunk(Ahi + tile, Ahi + F::T1 * F::A1_TILE + tile, tc::off_mnmajor(128, mb & 127, k1), re);
          tc_store_chunk(Ahi + tile, Ahi + F::T1 * F::A1_TILE + tile, tc::off_mnmajor(128, mb & 127, N1 + k1), im);
        }
      }
    }
  }
  if (!tc_gemm<K1, F::T1>(S, tmem, phase, S.A, F::A1_TILE, 1, S.B1, F::POLLS)) return false;

  // ---- D_B row (v, n2) holds conj(y[n2 + N2 n1]) / (rs sc_v), n1 < N1: stage
  // rows in shared memory (the operands are no longer read), then store them
  float2* stage = reinterpret_cast<float2*>(S.A);
  {
    const int t = warp >> 2;
    const int m = t * 128 + (warp & 3) * 32 + lane;
    const int v = m / N2, n2 = m - v * N2;
    float d[K1];
#pragma unroll
    for (int c = 0; c < K1; c += 16) tc::tmem_ld16(tmem + wl + t * K1 + c, d + c);
    tc::tmem_wait_ld();
    float mv = S.red[v];
#pragma unroll
    for (int w = 1; w < 8; ++w) mv = fmaxf(mv, S.red[w * 8 + v]);
    int e = 0;
    if (mv > 0.f) frexpf(mv, &e);
    const float back = ldexpf(1.f, e - 9 + LOG2N);  // undoes sc_v and rs
    // column-major staging (lanes hold consecutive n2 of one column): conflict-free
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) stage[v * N + n2 + N2 * n1] = make_float2(d[n1] * back, -d[N1 + n1] * back);
  }
  tc::fence_before_sync();
  __syncthreads();
  for (int n = tid; n < N; n += F::THREADS) {
    float2 row[8];
#pragma unroll
    for (int v = 0; v < 8; ++v) row[v] = stage[v * N + n];
    store_row(n, row);
  }
  __syncthreads();
  return true;
}

// Row FFTs of length N = L1 L2 (L1 = F::N1, L2 = F::N2) on eight rows: the
// same two GEMM stages, tile shapes, DFT matrices and shared-memory layout as
// the column form with the index maps exchanged, because a row's contiguous
// index must form the MN-major 16-byte chunks:
//   n = na + L2 nb (na < L2 contiguous, nb < L1),  k = L1 ka + kb,
//   X[L1 ka + kb] = sum_na W_L2^(na ka) W_N^(na kb) sum_nb W_L1^(nb kb) x[na + L2 nb].
// Stage 1 rows (v, na), a DFT of length L1 over nb; stage 2 rows (v, kb), a
// DFT of length L2 over na.  load8(v, n, out[8]): elements n .. n+7 of input
// row v (n a multiple of 8); store(v, k, X): output bin k of row v, staged
// through shared memory so rows leave contiguous.
// Each row is scaled by its own power of two.  STORE = false leaves the
// output in shared memory (tc_rows_staged: row v, bin k at [v N + k]) for the
// next call's loader, which reads all of it into registers before its first
// operand write; store is then not called.
template <class F, bool STORE = true, class Load8, class Store>
__device__ bool tc_fft_rows_tile(const TcFftSmem& S, uint32_t tmem, uint32_t& phase, const float2* __restrict__ tw,
                                 Load8 load8, Store store) {
  constexpr int L1 = F::N1, L2 = F::N2, N = F::N, K1 = F::K1, K2 = F::K2;
  constexpr int CPR = N / 8;  // 8-element chunks per row
  static_assert(L2 % 8 == 0, "a chunk of 8 shares nb");
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t wl = (uint32_t)((warp & 3) * 32) << 16;

  // ---- load: chunk c = tid + 256 i is row v = c / CPR; its 8 elements start at
  // n0 = 8 (r / L1) + L2 (r % L1), r = c % CPR (a chunk per (n_a group, n_b))
  float2 xv[F::RPT][8];
  float mx[8];
#pragma unroll
  for (int v = 0; v < 8; ++v) mx[v] = 0.f;
#pragma unroll
  for (int i = 0; i < F::RPT; ++i) {
    const int c = tid + i * F::THREADS;
    const int v = c / CPR, r = c - v * CPR;
    const int n0 = 8 * (r / L1) + L2 * (r % L1);  // nb = r % L1 fastest (conflict-free operand stores)
    load8(v, n0, xv[i]);
    float m = 0.f;
#pragma unroll
    for (int q = 0; q < 8; ++q) m = fmaxf(m, fmaxf(fabsf(xv[i][q].x), fabsf(xv[i][q].y)));
#pragma unroll
    for (int r = 0; r < 8; ++r) mx[r] = (r == v) ? fmaxf(mx[r], m) : mx[r];
  }
#pragma unroll
  for (int v = 0; v < 8; ++v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx[v] = fmaxf(mx[v], __shfl_xor_sync(0xffffffffu, mx[v], o));
  }
  if (lane == 0) {
#pragma unroll
    for (int v = 0; v < 8; ++v) S.red[warp * 8 + v] = mx[v];
  }
  __syncthreads();
  float sc[8];
#pragma unroll
  for (int v = 0; v < 8; ++v) {
    float m = S.red[v];
#pragma unroll
    for (int w = 1; w < 8; ++w) m = fmaxf(m, S.red[w * 8 + v]);
    int e = 0;
    if (m > 0.f) frexpf(m, &e);
    sc[v] = ldexpf(1.f, 9 - e);
  }

  // ---- stage-1 A (MN-major): row m = L2 v + na, column (re | im) of nb
  uint8_t* Ahi = S.A;
#pragma unroll
  for (int i = 0; i < F::RPT; ++i) {
    const int c = tid + i * F::THREADS;
    const int v = c / CPR, r = c - v * CPR;
    const int na0 = 8 * (r / L1), nb = r % L1;  // the chunk's 8 elements share nb (L2 % 8 == 0)
    float s = sc[0];
#pragma unroll
    for (int r = 1; r < 8; ++r) s = (r == v) ? sc[r] : s;
    float re[8], im[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      re[q] = xv[i][q].x * s;
      im[q] = xv[i][q].y * s;
    }
    const int m0 = v * L2 + na0;
    const uint32_t tile = (uint32_t)(m0 >> 7) * F::A1_TILE;
    tc_store_chunk(Ahi + tile, Ahi + F::T1 * F::A1_TILE + tile, tc::off_mnmajor(128, m0 & 127, nb), re);
    tc_store_chunk(Ahi + tile, Ahi + F::T1 * F::A1_TILE + tile, tc::off_mnmajor(128, m0 & 127, L1 + nb), im);
  }
  if (!tc_gemm<K1, F::T1>(S, tmem, phase, S.A, F::A1_TILE, 1, S.B1, F::POLLS)) return false;

  // ---- stage-1 result: thread = row (v, na); twiddle W_N^(na kb); stage-2 A
  // (MN-major): row (v, kb) = L1 v + kb, column (re | im) of na
  {
    const int t = warp >> 2;
    const int m = t * 128 + (warp & 3) * 32 + lane;
    const int v = m / L2, na = m - v * L2;
    float d[K1];
#pragma unroll
    for (int c = 0; c < K1; c += 16) tc::tmem_ld16(tmem + wl + t * K1 + c, d + c);
    tc::tmem_wait_ld();
#pragma unroll
    for (int c = 0; c < L1 / 8; ++c) {
      float re[8], im[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int kb = 8 * c + q;
        const float2 w = tw[na * kb];  // na kb < N
        re[q] = d[kb] * w.x - d[L1 + kb] * w.y;
        im[q] = d[kb] * w.y + d[L1 + kb] * w.x;
      }
      const int m2 = v * L1 + 8 * c;
      const uint32_t tile = (uint32_t)(m2 >> 7) * F::A2_TILE;
      tc_store_chunk(Ahi + tile, Ahi + F::T2 * F::A2_TILE + tile, tc::off_mnmajor(128, m2 & 127, na), re);
      tc_store_chunk(Ahi + tile, Ahi + F::T2 * F::A2_TILE + tile, tc::off_mnmajor(128, m2 & 127, L2 + na), im);
    }
  }
  if (!tc_gemm<K2, F::T2>(S, tmem, phase, S.A, F::A2_TILE, 1, S.B2, F::POLLS)) return false;

  // ---- stage-2 result: row (v, kb) holds X[L1 ka + kb], ka < L2; stage the
  // rows column-major by bin (lanes hold consecutive kb: conflict-free)
  float2* stage = reinterpret_cast<float2*>(S.A);
#pragma unroll
  for (int j0 = 0; j0 < F::T2; j0 += 2) {
    const int j = j0 + (warp >> 2);
    if (j < F::T2) {
      float d[K2];
#pragma unroll
      for (int c = 0; c < K2; c += 16) tc::tmem_ld16(tmem + wl + j * K2 + c, d + c);
      tc::tmem_wait_ld();
      const int m2 = j * 128 + (warp & 3) * 32 + lane;
      if (m2 < F::M2) {
        const int v = m2 / L1, kb = m2 - v * L1;
        float mv = S.red[v];
#pragma unroll
        for (int w = 1; w < 8; ++w) mv = fmaxf(mv, S.red[w * 8 + v]);
        int e = 0;
        if (mv > 0.f) frexpf(mv, &e);
        const float isc = ldexpf(1.f, e - 9);
        // the staged rows overwrite stage 2's operand, which the completed GEMM no longer reads
#pragma unroll
        for (int ka = 0; ka < L2; ++ka) stage[v * N + L1 * ka + kb] = make_float2(d[ka] * isc, d[L2 + ka] * isc);
      }
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if constexpr (STORE) {
    // lanes take consecutive bins: conflict-free reads, contiguous row stores
    for (int e = tid; e < 8 * N; e += F::THREADS) store(e / N, e % N, stage[e]);
    __syncthreads();
  }
  return true;
}

// the rows a tc_fft_rows_tile<F, false> call left in shared memory
__device__ __forceinline__ const float2* tc_rows_staged(const TcFftSmem& S) {
  return reinterpret_cast<const float2*>(S.A);
}

}  // namespace cx
