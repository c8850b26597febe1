// Register/shared-memory Stockham FFT engine for complex64 vectors.
//
// One "team" of LPV lanes transforms one length-N vector.  Each Stockham
// stage keeps its radix-R butterflies in registers; stages exchange data
// through a per-vector shared-memory buffer indexed with a one-in-sixteen
// skew (pad_idx) so that stride-R writes do not collide on banks.  The first
// stage pulls its inputs through a caller functor (global memory, a shared
// tile, or an analytic source) and the last stage hands its outputs to a
// caller functor (fused epilogue), so a pass costs one read and one write of
// the vector outside the engine.
//
// Mixed radix: N = 2^d 3^c 5^b 7^a: radix-16 stages and one of {2,4,8} (or
// 8*4) for the power of two, then the odd radices (see make_radices).  Twiddles exp(-2 pi i m / N) come from a table of N entries that each
// persistent CTA computes once in FP64 into shared memory.
#pragma once

#include "common.cuh"

namespace cx {

// ---------------------------------------------------------------------------
// compile-time plan
// ---------------------------------------------------------------------------
struct Radices {
  int n;
  int r[16];
};

__host__ __device__ constexpr Radices make_radices(int N) {
  // power-of-two radices first, odd radices last: with the n + n/16 skew every
  // stage's shared-memory exchange is then bank-conflict free (a stride-3/5/7
  // write in the first stage is not)
  Radices p{0, {0}};
  int m = N;
  int n7 = 0, n5 = 0, n3 = 0;
  while (m % 7 == 0) { ++n7; m /= 7; }
  while (m % 5 == 0) { ++n5; m /= 5; }
  while (m % 3 == 0) { ++n3; m /= 3; }
  int a = 0;
  while (m % 2 == 0) { m /= 2; ++a; }
  int n16 = a / 4, rem = a % 4;
  if (rem == 1 && n16 > 0) {
    for (int i = 0; i < n16 - 1; ++i) p.r[p.n++] = 16;
    p.r[p.n++] = 8;
    p.r[p.n++] = 4;
  } else {
    for (int i = 0; i < n16; ++i) p.r[p.n++] = 16;
    if (rem == 1) p.r[p.n++] = 2;
    if (rem == 2) p.r[p.n++] = 4;
    if (rem == 3) p.r[p.n++] = 8;
  }
  for (int i = 0; i < n3; ++i) p.r[p.n++] = 3;
  for (int i = 0; i < n5; ++i) p.r[p.n++] = 5;
  for (int i = 0; i < n7; ++i) p.r[p.n++] = 7;
  return p;
}

__host__ __device__ constexpr int max_radix(int N) {
  Radices p = make_radices(N);
  int mr = 1;
  for (int i = 0; i < p.n; ++i) mr = p.r[i] > mr ? p.r[i] : mr;
  return mr;
}

__host__ __device__ constexpr int pow2_floor(int v) {
  int p = 1;
  while (p * 2 <= v) p *= 2;
  return p;
}

// lanes per vector: one lane per butterfly of the largest-radix stage, so a
// lane holds about R_max complex values per stage.  Teams of up to 32 lanes
// live inside a warp (power-of-two size); larger teams are whole warps
// synchronised with a named barrier.
__host__ __device__ constexpr int lanes_per_vector(int N) {
  const int t = N / max_radix(N);
  if (t <= 32) {
    int l = 1;
    while (l < t) l *= 2;
    return l;
  }
  return ((t + 31) / 32) * 32;
}

__host__ __device__ constexpr int pad_idx(int n) { return n + (n >> 4); }
// per-vector shared-memory stride in float2 (odd, so column-tile transposes are bank-spread)
__host__ __device__ constexpr int vec_len(int N) {
  int l = pad_idx(N - 1) + 1;
  return (l % 2 == 0) ? l + 1 : l;
}

template <int N>
struct Plan {
  static constexpr Radices P = make_radices(N);
  static constexpr int S = P.n;
  static constexpr int LPV = lanes_per_vector(N);
  // one lane per butterfly of the largest-radix stage, without rounding to a
  // warp-friendly team size: teams of this size need CTA-wide barriers
  static constexpr int LPV_X = N / max_radix(N);
  static constexpr int LEN = vec_len(N);
  __host__ __device__ static constexpr int radix(int s) { return P.r[s]; }
  // outputs a lane holds after the last stage: the store functor's `slot`
  // argument (compile-time after unrolling) indexes [0, OUT_SLOTS)
  static constexpr int R_LAST = P.r[P.n - 1];
  static constexpr int OUT_SLOTS = ((N / R_LAST + LPV - 1) / LPV) * R_LAST;
};

// ---------------------------------------------------------------------------
// small DFTs (forward: exp(-2 pi i rk/R); INV: exp(+2 pi i rk/R))
// ---------------------------------------------------------------------------
template <bool INV>
__device__ __forceinline__ void dft2(float2& a, float2& b) {
  float2 t = a;
  a = cadd(t, b);
  b = csub(t, b);
}

template <bool INV>
__device__ __forceinline__ void dft4(float2& x0, float2& x1, float2& x2, float2& x3) {
  float2 t0 = cadd(x0, x2), t1 = csub(x0, x2), t2 = cadd(x1, x3), t3 = mul_mi<INV>(csub(x1, x3));
  x0 = cadd(t0, t2);
  x2 = csub(t0, t2);
  x1 = cadd(t1, t3);
  x3 = csub(t1, t3);
}

template <int R, bool INV>
struct DFT;

template <bool INV>
struct DFT<2, INV> {
  __device__ __forceinline__ static void run(float2* v) { dft2<INV>(v[0], v[1]); }
};

template <bool INV>
struct DFT<4, INV> {
  __device__ __forceinline__ static void run(float2* v) { dft4<INV>(v[0], v[1], v[2], v[3]); }
};

template <bool INV>
struct DFT<8, INV> {
  __device__ __forceinline__ static void run(float2* v) {
    const float h = 0.70710678118654752440f;
    // r = r1 + 2 r2 ; DFT4 over r2 for r1 = 0, 1
    dft4<INV>(v[0], v[2], v[4], v[6]);
    dft4<INV>(v[1], v[3], v[5], v[7]);
    // twiddles w8^(r1*k2) for r1 = 1, k2 = 1..3
    float2 a1 = v[3], a2 = v[5], a3 = v[7];
    // w8^1 = (h, -h) fwd ; (h, +h) inv
    v[3] = INV ? make_float2(h * (a1.x - a1.y), h * (a1.x + a1.y)) : make_float2(h * (a1.x + a1.y), h * (a1.y - a1.x));
    v[5] = mul_mi<INV>(a2);
    // w8^3 = (-h, -h) fwd ; (-h, +h) inv
    v[7] = INV ? make_float2(-h * (a3.x + a3.y), h * (a3.x - a3.y)) : make_float2(h * (a3.y - a3.x), -h * (a3.x + a3.y));
    // DFT2 over r1 ; output k = k2 + 4 k1
    float2 y[8];
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) {
      float2 p = v[2 * k2], q = v[2 * k2 + 1];
      y[k2] = cadd(p, q);
      y[k2 + 4] = csub(p, q);
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = y[i];
  }
};

template <bool INV>
struct DFT<16, INV> {
  __device__ __forceinline__ static void run(float2* v) {
    const float c1 = 0.92387953251128675613f;  // cos(pi/8)
    const float s1 = 0.38268343236508977173f;  // sin(pi/8)
    const float h = 0.70710678118654752440f;
    const float sg = INV ? 1.f : -1.f;
    // r = r1 + 4 r2 ; DFT4 over r2 for each r1
#pragma unroll
    for (int r1 = 0; r1 < 4; ++r1) dft4<INV>(v[r1], v[r1 + 4], v[r1 + 8], v[r1 + 12]);
    // a[r1][k2] = v[r1 + 4 k2]; twiddle w16^(r1*k2)
    // r1 = 1: k2 = 1,2,3 -> w^1, w^2, w^3
    v[5] = cmul(v[5], make_float2(c1, sg * s1));
    v[9] = cmul(v[9], make_float2(h, sg * h));
    v[13] = cmul(v[13], make_float2(s1, sg * c1));
    // r1 = 2: w^2, w^4, w^6
    v[6] = cmul(v[6], make_float2(h, sg * h));
    v[10] = mul_mi<INV>(v[10]);
    v[14] = cmul(v[14], make_float2(-h, sg * h));
    // r1 = 3: w^3, w^6, w^9
    v[7] = cmul(v[7], make_float2(s1, sg * c1));
    v[11] = cmul(v[11], make_float2(-h, sg * h));
    v[15] = cmul(v[15], make_float2(-c1, -sg * s1));
    // DFT4 over r1 for each k2 ; output k = k2 + 4 k1
    float2 y[16];
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) {
      float2 a0 = v[4 * k2 + 0], a1 = v[4 * k2 + 1], a2 = v[4 * k2 + 2], a3 = v[4 * k2 + 3];
      dft4<INV>(a0, a1, a2, a3);
      y[k2] = a0;
      y[k2 + 4] = a1;
      y[k2 + 8] = a2;
      y[k2 + 12] = a3;
    }
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = y[i];
  }
};

// odd prime radices via symmetric pairs:
// y_k = x0 + sum_m [ (x_m + x_{R-m}) cos(2 pi k m/R) -/+ i (x_m - x_{R-m}) sin(2 pi k m/R) ]
template <int R>
struct OddConst;
template <>
struct OddConst<3> {
  __device__ static constexpr float c(int i) { return -0.5f; }
  __device__ static constexpr float s(int i) { return 0.86602540378443864676f; }
};
template <>
struct OddConst<5> {
  __device__ static constexpr float c(int i) {
    return i == 1 ? 0.30901699437494742410f : (i == 2 ? -0.80901699437494742410f : 0.f);
  }
  __device__ static constexpr float s(int i) {
    return i == 1 ? 0.95105651629515357212f : (i == 2 ? 0.58778525229247312917f : 0.f);
  }
};
template <>
struct OddConst<7> {
  __device__ static constexpr float c(int i) {
    return i == 1 ? 0.62348980185873353053f : (i == 2 ? -0.22252093395631440429f : (i == 3 ? -0.90096886790241912624f : 0.f));
  }
  __device__ static constexpr float s(int i) {
    return i == 1 ? 0.78183148246802980871f : (i == 2 ? 0.97492791218182360702f : (i == 3 ? 0.43388373911755812048f : 0.f));
  }
};

template <int R, bool INV>
struct DFTOdd {
  __device__ __forceinline__ static void run(float2* v) {
    constexpr int H = (R - 1) / 2;
    float2 sp[H + 1], dm[H + 1];
#pragma unroll
    for (int m = 1; m <= H; ++m) {
      sp[m] = cadd(v[m], v[R - m]);
      dm[m] = csub(v[m], v[R - m]);
    }
    float2 y0 = v[0];
#pragma unroll
    for (int m = 1; m <= H; ++m) y0 = cadd(y0, sp[m]);
    float2 out[R];
    out[0] = y0;
#pragma unroll
    for (int k = 1; k <= H; ++k) {
      float2 re = v[0];
      float2 im = make_float2(0.f, 0.f);
#pragma unroll
      for (int m = 1; m <= H; ++m) {
        const int idx = (k * m) % R;  // cos(2 pi idx/R) ; sin sign from symmetry
        const int ii = idx <= H ? idx : R - idx;
        const float c = OddConst<R>::c(ii);
        const float s = (idx <= H ? 1.f : -1.f) * OddConst<R>::s(ii);
        re = make_float2(re.x + c * sp[m].x, re.y + c * sp[m].y);
        im = make_float2(im.x + s * dm[m].x, im.y + s * dm[m].y);
      }
      // forward: -i * im ; inverse: +i * im
      float2 t = mul_mi<INV>(im);
      out[k] = cadd(re, t);
      out[R - k] = csub(re, t);
    }
#pragma unroll
    for (int i = 0; i < R; ++i) v[i] = out[i];
  }
};
template <bool INV>
struct DFT<3, INV> : DFTOdd<3, INV> {};
template <bool INV>
struct DFT<5, INV> {
  __device__ __forceinline__ static void run(float2* v) {
    const float c1 = 0.30901699437494742410f, c2 = -0.80901699437494742410f;  // cos(2pi/5), cos(4pi/5)
    const float s1 = 0.95105651629515357212f, s2 = 0.58778525229247312917f;   // sin(2pi/5), sin(4pi/5)
    const float2 a1 = cadd(v[1], v[4]), b1 = csub(v[1], v[4]);
    const float2 a2 = cadd(v[2], v[3]), b2 = csub(v[2], v[3]);
    const float2 x0 = v[0];
    v[0] = make_float2(x0.x + a1.x + a2.x, x0.y + a1.y + a2.y);
    const float2 r1 = make_float2(x0.x + c1 * a1.x + c2 * a2.x, x0.y + c1 * a1.y + c2 * a2.y);
    const float2 r2 = make_float2(x0.x + c2 * a1.x + c1 * a2.x, x0.y + c2 * a1.y + c1 * a2.y);
    const float2 i1 = make_float2(s1 * b1.x + s2 * b2.x, s1 * b1.y + s2 * b2.y);
    const float2 i2 = make_float2(s2 * b1.x - s1 * b2.x, s2 * b1.y - s1 * b2.y);
    const float2 t1 = mul_mi<INV>(i1), t2 = mul_mi<INV>(i2);
    v[1] = cadd(r1, t1);
    v[4] = csub(r1, t1);
    v[2] = cadd(r2, t2);
    v[3] = csub(r2, t2);
  }
};

template <bool INV>
struct DFT<7, INV> : DFTOdd<7, INV> {};

// ---------------------------------------------------------------------------
// team synchronisation
// ---------------------------------------------------------------------------
template <int LPV>
__device__ __forceinline__ void team_sync(int team) {
  if constexpr (LPV < 32) {
    // only this team's lanes: teams sharing a warp may take different paths
    const unsigned base = ((threadIdx.x & 31u) / LPV) * LPV;
    __syncwarp(((LPV == 32 ? 0u : (1u << LPV)) - 1u) << base);
  } else if constexpr (LPV == 32) {
    __syncwarp();
  } else {
    // named barrier per team (ids 1..15); team = threadIdx.x / LPV
    asm volatile("bar.sync %0, %1;" ::"r"(1 + team), "r"(LPV) : "memory");
  }
}

// Team barrier: team-local (CTA = false) or CTA-wide (CTA = true, for teams
// that do not tile warps; every thread of the CTA must then reach it)
template <int LPV, bool CTA>
__device__ __forceinline__ void team_barrier(int team) {
  if constexpr (CTA) {
    __syncthreads();
  } else {
    team_sync<LPV>(team);
  }
}

// ---------------------------------------------------------------------------
// twiddle table: tw[m] = exp(-2 pi i m / N), computed in FP64
// ---------------------------------------------------------------------------
// table length: tw[m] = w^m for m < N, then tw[N + m] = w^(4m) for m < N/8
__host__ __device__ constexpr int tw_len(int N) { return N + N / 8 + 1; }

// exp(-2 pi i e / N), e in [0, N): for N divisible by 8 only the first octant
// is evaluated (FP64 sincospi) and the rest follows by exact symmetries
template <int N>
__device__ __forceinline__ float2 twiddle_value(int e) {
  if constexpr (N % 8 == 0) {
    constexpr int Q = N / 4, O = N / 8;
    const int q = e / Q, r = e - q * Q;  // e = q N/4 + r, 0 <= r < N/4
    const bool hi = r > O;               // second octant of the quadrant: mirror
    const int m = hi ? Q - r : r;        // 0 <= m <= N/8
    double sd, cd;
    sincospi(2.0 * (double)m / (double)N, &sd, &cd);
    // angle t = 2 pi r / N ; (cos t, sin t)
    float c = hi ? (float)sd : (float)cd;
    float sn = hi ? (float)cd : (float)sd;
    // rotate by q quarter turns: exp(i (t + q pi/2))
    float cr = c, sr = sn;
    if (q == 1) { cr = -sn; sr = c; }
    if (q == 2) { cr = -c; sr = -sn; }
    if (q == 3) { cr = sn; sr = -c; }
    return make_float2(cr, -sr);  // exp(-i angle)
  } else {
    double sd, cd;
    sincospi(-2.0 * (double)e / (double)N, &sd, &cd);
    return make_float2((float)cd, (float)sd);
  }
}

template <int N>
__device__ __forceinline__ void init_twiddles(float2* tw, int tid, int nthreads) {
  for (int m = tid; m < tw_len(N); m += nthreads) {
    const int e = m < N ? m : (4 * (m - N)) % N;
    tw[m] = twiddle_value<N>(e);
  }
}

// v[r] *= exp(-/+ 2 pi i r m / N) for 0 < r < R.  At most two table loads
// (tw[m], tw[4m]); the other factors are products of at most three table
// values, applied as they are formed so few twiddles are live at once.
template <int R, bool INV, int N>
__device__ __forceinline__ void apply_twiddles(const float2* tw, int m, float2* v) {
  float2 w1 = tw[m];
  if (INV) w1.y = -w1.y;
  v[1] = cmul(v[1], w1);
  if constexpr (R >= 3) {
    const float2 w2 = cmul(w1, w1);
    v[2] = cmul(v[2], w2);
    if constexpr (R >= 4) {
      const float2 w3 = cmul(w2, w1);
      v[3] = cmul(v[3], w3);
      if constexpr (R == 5 || R == 7) {
        const float2 w4 = cmul(w2, w2);
        v[4] = cmul(v[4], w4);
        if constexpr (R == 7) {
          v[5] = cmul(v[5], cmul(w4, w1));
          v[6] = cmul(v[6], cmul(w4, w2));
        }
      }
      if constexpr (R == 8 || R == 16) {
        float2 w4 = tw[N + m];  // contiguous copy of tw[4 m] (bank-conflict free)
        if (INV) w4.y = -w4.y;
        v[4] = cmul(v[4], w4);
        v[5] = cmul(v[5], cmul(w4, w1));
        v[6] = cmul(v[6], cmul(w4, w2));
        v[7] = cmul(v[7], cmul(w4, w3));
        if constexpr (R == 16) {
          const float2 w8 = cmul(w4, w4);
          v[8] = cmul(v[8], w8);
          v[9] = cmul(v[9], cmul(w8, w1));
          v[10] = cmul(v[10], cmul(w8, w2));
          v[11] = cmul(v[11], cmul(w8, w3));
          const float2 w12 = cmul(w8, w4);
          v[12] = cmul(v[12], w12);
          v[13] = cmul(v[13], cmul(w12, w1));
          v[14] = cmul(v[14], cmul(w12, w2));
          v[15] = cmul(v[15], cmul(w12, w3));
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// the stage recursion
// ---------------------------------------------------------------------------
// ZM (first stage only): bit r set = inputs j + r N/R_0 are known to be zero
// for every j, so they are compile-time zeros and their arithmetic folds away
template <int N, int LPV, bool INV, int SI, int NS, bool CTA = false, unsigned ZM = 0u>
struct Stage {
  static constexpr int S = Plan<N>::S;
  static constexpr int R = Plan<N>::radix(SI);
  static constexpr int NBF = N / R;
  static constexpr int IT = (NBF + LPV - 1) / LPV;
  static constexpr bool FIRST = (SI == 0);
  static constexpr bool LAST = (SI == S - 1);
  static constexpr bool EXACT = (NBF % LPV) == 0;

  template <class Load, class Store>
  __device__ __forceinline__ static void run(float2* s, const float2* tw, int lane, int team, Load& load,
                                             Store& store) {
    float2 v[IT][R];
#pragma unroll
    for (int it = 0; it < IT; ++it) {
      // Lanes past the last butterfly recompute the last one (in bounds) and
      // never store it: keeping the compute branch-free lets ptxas schedule
      // the stage with far fewer live registers than a guarded block.
      const int j = (EXACT || lane + it * LPV < NBF) ? lane + it * LPV : NBF - 1;
      {
        if constexpr (FIRST) {
#pragma unroll
          for (int r = 0; r < R; ++r) v[it][r] = ((ZM >> r) & 1u) ? make_float2(0.f, 0.f) : load(j + r * NBF);
        } else if constexpr (NBF % 16 == 0) {
          // pad_idx(j + r NBF) = pad_idx(j) + r (NBF + NBF/16): one address,
          // immediate offsets
          const float2* sp = s + pad_idx(j);
#pragma unroll
          for (int r = 0; r < R; ++r) v[it][r] = sp[r * (NBF + NBF / 16)];
        } else {
#pragma unroll
          for (int r = 0; r < R; ++r) v[it][r] = s[pad_idx(j + r * NBF)];
        }
        if constexpr (!FIRST) {
          const int k = j % NS;
          constexpr int TS = N / (NS * R);
          apply_twiddles<R, INV, N>(tw, k * TS, v[it]);
        }
        DFT<R, INV>::run(v[it]);
      }
    }
    if constexpr (LAST) {
      // the store functor may write the team's buffer that this stage read
      team_barrier<LPV, CTA>(team);
#pragma unroll
      for (int it = 0; it < IT; ++it) {
        const int j = lane + it * LPV;
        if (EXACT || j < NBF) {
#pragma unroll
          for (int r = 0; r < R; ++r) store(j + r * NBF, v[it][r], it * R + r);
        }
      }
    } else {
      team_barrier<LPV, CTA>(team);
#pragma unroll
      for (int it = 0; it < IT; ++it) {
        const int j = lane + it * LPV;
        if (EXACT || j < NBF) {
          const int k = j % NS;
          const int base = (j - k) * R + k;
          if constexpr (NS % 16 == 0) {
            float2* sp = s + pad_idx(base);
#pragma unroll
            for (int r = 0; r < R; ++r) sp[r * (NS + NS / 16)] = v[it][r];
          } else if constexpr (NS == 1 && 16 % R == 0) {
            // base = j R is a multiple of R, so base + r (r < R) stays in one
            // run of 16 and pad_idx(base + r) = pad_idx(base) + r
            float2* sp = s + pad_idx(base);
#pragma unroll
            for (int r = 0; r < R; ++r) sp[r] = v[it][r];
          } else {
#pragma unroll
            for (int r = 0; r < R; ++r) s[pad_idx(base + r * NS)] = v[it][r];
          }
        }
      }
      team_barrier<LPV, CTA>(team);
      Stage<N, LPV, INV, SI + 1, NS * R, CTA>::run(s, tw, lane, team, load, store);
    }
  }
};

// terminate recursion past the last stage (never instantiated at run time)
template <int N, int LPV, bool INV, int NS, bool CTA, unsigned ZM>
struct Stage<N, LPV, INV, 16, NS, CTA, ZM> {
  template <class Load, class Store>
  __device__ static void run(float2*, const float2*, int, int, Load&, Store&) {}
};

// Transform one vector.  `s` is the team's shared buffer of Plan<N>::LEN
// float2; `load(n)` returns input n, `store(k, v, slot)` consumes output k
// (`slot` in [0, Plan<N>::OUT_SLOTS) identifies the lane's output
// register, for per-lane accumulation across calls).  All
// lanes of the team must call this (inactive lanes still take part in the
// team barriers).  Outputs are unnormalised (numpy convention for the
// forward transform; the inverse omits the 1/N).
template <int N, bool INV, int LPV = Plan<N>::LPV, bool CTA = false, unsigned ZM = 0u, class Load, class Store>
__device__ __forceinline__ void team_fft(float2* s, const float2* tw, int lane, int team, Load& load, Store& store) {
  Stage<N, LPV, INV, 0, 1, CTA, ZM>::run(s, tw, lane, team, load, store);
}

// Zero mask for team_fft when the input vector is nonzero only on
// [0, h) and [N - h, N) with h <= Q N / R_0 (a centred support after an
// ifftshift): first-stage inputs r in [Q, R_0 - Q) are zero.
template <int N, int Q>
__host__ __device__ constexpr unsigned edge_zero_mask() {
  constexpr int R0 = Plan<N>::P.r[0];
  unsigned m = 0u;
  for (int r = Q; r < R0 - Q; ++r) m |= 1u << r;
  return m;
}

// First-stage zero mask for an input that is nonzero only on the central
// band [N / 4, 3 N / 4) (a field zero-padded to twice its size on both
// sides): with a first radix R_0 divisible by 4, the inputs j + r N / R_0 with
// r < R_0 / 4 or r >= 3 R_0 / 4 are zero.  0 (no mask) otherwise.
template <int N>
__host__ __device__ constexpr unsigned center_band_mask() {
  constexpr int R0 = Plan<N>::P.r[0];
  unsigned m = 0u;
  if (R0 % 4 == 0)
    for (int r = 0; r < R0; ++r)
      if (r < R0 / 4 || r >= 3 * R0 / 4) m |= 1u << r;
  return m;
}

// First-stage zero mask for an input that is nonzero only on [0, N / 2)
// (zero padding to twice the length): with an even first radix R_0 the
// inputs r >= R_0 / 2 of every first-stage butterfly (indices
// j + r N / R_0 >= N / 2) are zero.  Odd first radices (odd N) get no mask.
template <int N>
__host__ __device__ constexpr unsigned lower_half_mask() {
  constexpr int R0 = Plan<N>::P.r[0];
  unsigned m = 0u;
  if (R0 % 2 == 0)
    for (int r = R0 / 2; r < R0; ++r) m |= 1u << r;
  return m;
}

// Same transform with the load and/or store functor applied in a compact,
// coalesced loop through the team's shared buffer (lane-strided indices)
// instead of once per butterfly value inside the unrolled first / last
// stage.  Costs one extra shared-memory pass per staged side but emits the
// functor's code once: for heavy functors (FP64 phase evaluation, sin/cos,
// transmittances) this keeps the kernel within the instruction cache.
// Staged store functors receive slot = 0.
template <int N, bool INV, bool STAGE_LOAD, bool STAGE_STORE, int LPV = Plan<N>::LPV, bool CTA = false,
          unsigned ZM = 0u, class Load, class Store>
__device__ __forceinline__ void team_fft_ex(float2* s, const float2* tw, int lane, int team, Load& load,
                                            Store& store) {
  auto sld = [&](int n) -> float2 { return s[pad_idx(n)]; };
  auto sst = [&](int k, float2 v, int) { s[pad_idx(k)] = v; };
  if constexpr (STAGE_LOAD) {
    team_barrier<LPV, CTA>(team);  // the previous use of the buffer is complete
#pragma unroll 4
    for (int n = lane; n < N; n += LPV) s[pad_idx(n)] = load(n);
    team_barrier<LPV, CTA>(team);
    if constexpr (STAGE_STORE) {
      Stage<N, LPV, INV, 0, 1, CTA>::run(s, tw, lane, team, sld, sst);
    } else {
      Stage<N, LPV, INV, 0, 1, CTA>::run(s, tw, lane, team, sld, store);
    }
  } else {
    // ZM (first-stage zero mask) applies to the caller's loads only
    if constexpr (STAGE_STORE) {
      Stage<N, LPV, INV, 0, 1, CTA, ZM>::run(s, tw, lane, team, load, sst);
    } else {
      Stage<N, LPV, INV, 0, 1, CTA, ZM>::run(s, tw, lane, team, load, store);
    }
  }
  if constexpr (STAGE_STORE) {
    team_barrier<LPV, CTA>(team);
#pragma unroll 2
    for (int k = lane; k < N; k += LPV) store(k, s[pad_idx(k)], 0);
  }
}

}  // namespace cx
