// Polarized (birefringent) thick sample, polarized_multislice_thick_sample
// (functional/samples.py:444-546), for a monochromatic vector field u
// (ny, nx, 3), components (z, y, x), on the zero-padded (2 ny, 2 nx) grid:
//   U = FFT2(pad u);  a = crop IFFT2(Q U);  s = V_i a;  S = FFT2(pad s)
//   u <- crop IFFT2(Q (e U + h S))      (= P_op(u) + H_op(s), one inverse)
// Q = I - k k^T / km^2 with k = (kz, ky, kx), zero outside |k_perp| <= NA km;
// e = exp(i kz dz), h = -i/2 exp(i kz dz) dz / kz (both 0 where kz = 0).
// Per slice two row passes and two column passes; the teams of a CTA hold
// the three components of a row / a column tile, so the 3x3 mixing runs in
// shared memory between the transforms.
#include <cmath>

#include "host.cuh"

namespace cx {

enum PolMode { POL_LOAD = 0, POL_SCATTER = 1, POL_NEXT = 2 };

struct PolArgs {
  int N, M, P, Q;             // field (N, M), padded (P, Q) = (2N, 2M)
  int mode, last, slice;
  int n_wv, wv;               // wavelengths interleaved in u_in / u_out, the one processed
  double km, NA2km2, dy, dx;  // km = 2 pi n / lambda
  float scale;                // 1 / (P Q)
  const float2* u_in;         // (N, M, W, 3)
  float2* u_out;              // (N, M, W, 3)
  const float* V;             // (D, N, M, 3, 3) potential
  const float2* Tin;          // (N, Q, 3) x-spectra
  float2* Tout;               // (N, Q, 3)
  float2* W;                  // (P, Q, 3) e U
  const float4* EH;           // (P, Q) {e, h}
  const float2* twg;
};

// ---------------------------------------------------------------------------
// rows: a CTA holds R rows x 3 components (one team each)
// ---------------------------------------------------------------------------
// about 96 threads (3 teams of 32 lanes at Q = 512): a 256-row field then runs
// 256 CTAs instead of 64
template <int Q>
struct PolRowCfg {
  static constexpr int LPV = Plan<Q>::LPV;
  static constexpr int R0 = 32 / LPV > 0 ? 32 / LPV : 1;
  static constexpr int R = LPV >= 32 && R0 > 5 ? 5 : R0;  // named barriers 1..15
  static constexpr int TEAMS = 3 * R;
  static constexpr int THREADS = TEAMS * LPV;
  static_assert(THREADS <= 1024, "polarized row CTA");
  static constexpr int LEN = Plan<Q>::LEN;
  static constexpr int TW = tw_len(Q);
  static constexpr int MINB = minb_for(THREADS);
  static constexpr size_t SMEM = sizeof(float2) * ((size_t)TW + (size_t)TEAMS * LEN);
};

template <int Q, int MODE>
__global__ void __launch_bounds__(PolRowCfg<Q>::THREADS, PolRowCfg<Q>::MINB) k_pol_rows(PolArgs a) {
  using C = PolRowCfg<Q>;
  constexpr int LPV = C::LPV, R = C::R;
  extern __shared__ float2 sm[];
  float2* tw = sm;
  load_twiddles<Q>(tw, a.twg, threadIdx.x, blockDim.x);
  __syncthreads();
  const int team = threadIdx.x / LPV, lane = threadIdx.x % LPV;
  const int r = team / 3, c = team % 3;
  float2* bufs = sm + C::TW;
  float2* s = bufs + team * C::LEN;
  auto sst = [&](int k, float2 v, int) { s[pad_idx(k)] = v; };
  for (int base = blockIdx.x * R; base < a.N; base += gridDim.x * R) {  // uniform over the CTA
    const int y = base + r;
    const bool valid = y < a.N;
    if constexpr (MODE == POL_LOAD) {
      if (valid) {
        const size_t es = (size_t)a.n_wv * 3;  // element stride
        const float2* src = a.u_in + (size_t)y * a.M * es + (size_t)a.wv * 3 + c;
        auto load = [&](int n) -> float2 { return n < a.M ? src[(size_t)n * es] : make_float2(0.f, 0.f); };
        float2* dst = a.Tout + (size_t)y * Q * 3 + c;
        auto store = [&](int k, float2 v, int) { dst[(size_t)k * 3] = v; };
        team_fft<Q, false, LPV, false, lower_half_mask<Q>()>(s, tw, lane, team, load, store);
      }
      continue;
    }
    if (valid) {
      const float2* src = a.Tin + (size_t)y * Q * 3 + c;
      auto load = [&](int n) -> float2 { return src[(size_t)n * 3]; };
      team_fft<Q, true, LPV>(s, tw, lane, team, load, sst);
    }
    __syncthreads();
    // pointwise over the row's three components: the threads of row r's teams
    {
      const int t3 = threadIdx.x - r * 3 * LPV;  // 0 .. 3 LPV - 1
      float2* s0 = bufs + (3 * r) * C::LEN;
      float2* s1 = s0 + C::LEN;
      float2* s2 = s1 + C::LEN;
      const float* Vr = MODE == POL_SCATTER ? a.V + ((size_t)a.slice * a.N + (valid ? y : 0)) * a.M * 9 : nullptr;
      const size_t es = (size_t)a.n_wv * 3;
      float2* orow = (MODE == POL_NEXT && a.last) ? a.u_out + (size_t)(valid ? y : 0) * a.M * es + (size_t)a.wv * 3
                                                    : nullptr;
      for (int x = t3; x < Q && valid; x += 3 * LPV) {
        const int px = pad_idx(x);
        if (x >= a.M) {
          s0[px] = s1[px] = s2[px] = make_float2(0.f, 0.f);
          continue;
        }
        float2 v0 = cscale(s0[px], a.scale), v1 = cscale(s1[px], a.scale), v2 = cscale(s2[px], a.scale);
        if constexpr (MODE == POL_SCATTER) {
          const float* m = Vr + (size_t)x * 9;  // rows (z, y, x) of the 3x3 potential
          const float2 w0 = make_float2(m[0] * v0.x + m[1] * v1.x + m[2] * v2.x, m[0] * v0.y + m[1] * v1.y + m[2] * v2.y);
          const float2 w1 = make_float2(m[3] * v0.x + m[4] * v1.x + m[5] * v2.x, m[3] * v0.y + m[4] * v1.y + m[5] * v2.y);
          const float2 w2 = make_float2(m[6] * v0.x + m[7] * v1.x + m[8] * v2.x, m[6] * v0.y + m[7] * v1.y + m[8] * v2.y);
          v0 = w0;
          v1 = w1;
          v2 = w2;
        }
        if (orow) {
          orow[(size_t)x * es + 0] = v0;
          orow[(size_t)x * es + 1] = v1;
          orow[(size_t)x * es + 2] = v2;
        }
        s0[px] = v0;
        s1[px] = v1;
        s2[px] = v2;
      }
    }
    __syncthreads();
    if (valid && !(MODE == POL_NEXT && a.last)) {
      auto load = [&](int n) -> float2 { return s[pad_idx(n)]; };
      float2* dst = a.Tout + (size_t)y * Q * 3 + c;
      auto store = [&](int k, float2 v, int) { dst[(size_t)k * 3] = v; };
      team_fft<Q, false, LPV, false, lower_half_mask<Q>()>(s, tw, lane, team, load, store);
    }
    __syncthreads();  // the buffers are reused by the next rows
  }
}

// ---------------------------------------------------------------------------
// columns: a CTA holds V spectrum columns x 3 components (3V teams)
// ---------------------------------------------------------------------------
template <int P>
struct PolColCfg {
  static constexpr int LPV = Plan<P>::LPV;
  static constexpr int TW = tw_len(P);
  static constexpr size_t smem_for(int v) { return sizeof(float2) * ((size_t)TW + 3 * (size_t)v * col_len(P, 3 * v)); }
  static constexpr int pick() {
    int v = 16;
    while (v > 1 && (3 * v * LPV > 768 || (LPV >= 32 && 3 * v > 15) || smem_for(v) > 200 * 1024)) v /= 2;
    return v;
  }
  static constexpr int V = pick();
  static constexpr int TEAMS = 3 * V;
  static constexpr int THREADS = TEAMS * LPV;
  static_assert(THREADS <= 1024 && (LPV < 32 || TEAMS <= 15), "polarized column CTA");
  static constexpr int LEN = col_len(P, 3 * V);
  static constexpr int MINB = 1;
  static constexpr size_t SMEM = smem_for(V);
};

// MODE: 1 = first column pass (A = Q U, W = e U), 2 = second (X = Q (W + h S))
template <int P, int MODE>
__global__ void __launch_bounds__(PolColCfg<P>::THREADS, PolColCfg<P>::MINB) k_pol_cols(PolArgs a) {
  using C = PolColCfg<P>;
  constexpr int V = C::V, LEN = C::LEN, LPV = C::LPV, TV = 3 * V;
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* tile = sm + C::TW;
  load_twiddles<P>(tw, a.twg, threadIdx.x, blockDim.x);
  const int team = threadIdx.x / LPV, lane = threadIdx.x % LPV;
  float2* s = tile + team * LEN;
  const int Q = a.Q;
  const int tiles = (Q + V - 1) / V;
  const float inv_km = (float)(1.0 / a.km);
  for (int t = blockIdx.x; t < tiles; t += gridDim.x) {
    const int kx0 = t * V;
    __syncthreads();
    load_col_tile<TV, LEN>(tile, a.Tin, (size_t)Q * 3, 3 * kx0, 3 * Q, 0, a.N, [](int rr) { return rr; });
    __syncthreads();
    {
      auto load = [&](int n) -> float2 { return n < a.N ? s[pad_idx(n)] : make_float2(0.f, 0.f); };
      auto store = [&](int k, float2 v, int) { s[pad_idx(k)] = v; };
      team_fft<P, false, LPV, false, lower_half_mask<P>()>(s, tw, lane, team, load, store);
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < P * V; idx += blockDim.x) {
      const int ky = idx / V, cj = idx % V, kx = kx0 + cj;
      if (kx >= Q) continue;
      const int pk = pad_idx(ky);
      float2* t0 = tile + (3 * cj) * LEN + pk;
      float2* t1 = t0 + LEN;
      float2* t2 = t1 + LEN;
      // FP64 |k_perp|^2 and kz: km^2 - |k_perp|^2 cancels near the evanescent boundary
      const double kyd = 6.283185307179586 * freq_index(ky, P) / (P * a.dy);
      const double kxd = 6.283185307179586 * freq_index(kx, Q) / (Q * a.dx);
      const double kp2 = kyd * kyd + kxd * kxd;
      const size_t wi = ((size_t)ky * Q + kx) * 3;
      float2 x0, x1, x2;
      if constexpr (MODE == 1) {
        const float4 eh = a.EH[(size_t)ky * Q + kx];
        const float2 e = make_float2(eh.x, eh.y);
        x0 = *t0;
        x1 = *t1;
        x2 = *t2;
        a.W[wi + 0] = cmul(e, x0);
        a.W[wi + 1] = cmul(e, x1);
        a.W[wi + 2] = cmul(e, x2);
      } else {
        const float4 eh = a.EH[(size_t)ky * Q + kx];
        const float2 h = make_float2(eh.z, eh.w);
        x0 = cadd(a.W[wi + 0], cmul(h, *t0));
        x1 = cadd(a.W[wi + 1], cmul(h, *t1));
        x2 = cadd(a.W[wi + 2], cmul(h, *t2));
      }
      float2 y0 = make_float2(0.f, 0.f), y1 = y0, y2 = y0;
      if (kp2 <= a.NA2km2) {
        // Q = I - k k^T / km^2, k = (kz, ky, kx), kz = sqrt(max(km^2 - |k_perp|^2, 0))
        const float k0 = (float)(sqrt(fmax(a.km * a.km - kp2, 0.0)) / a.km);
        const float k1 = (float)kyd * inv_km, k2 = (float)kxd * inv_km;
        const float d0 = k0 * x0.x + k1 * x1.x + k2 * x2.x, di = k0 * x0.y + k1 * x1.y + k2 * x2.y;
        y0 = make_float2(x0.x - k0 * d0, x0.y - k0 * di);
        y1 = make_float2(x1.x - k1 * d0, x1.y - k1 * di);
        y2 = make_float2(x2.x - k2 * d0, x2.y - k2 * di);
      }
      *t0 = y0;
      *t1 = y1;
      *t2 = y2;
    }
    __syncthreads();
    {
      auto load = [&](int n) -> float2 { return s[pad_idx(n)]; };
      auto store = [&](int k, float2 v, int) { s[pad_idx(k)] = v; };
      team_fft<P, true, LPV>(s, tw, lane, team, load, store);
    }
    __syncthreads();
    // rows < N of the 3V columns
    for (int idx = threadIdx.x; idx < a.N * TV; idx += blockDim.x) {
      const int rr = idx / TV, j = idx % TV, col = 3 * kx0 + j;
      if (col < 3 * Q) a.Tout[(size_t)rr * Q * 3 + col] = tile[j * LEN + pad_idx(rr)];
    }
  }
}

// e = exp(i kz dz), h = -i/2 exp(i kz dz) dz / kz (0 where kz = 0), FP64
__global__ void k_pol_table(float4* __restrict__ EH, int P, int Q, double km, double dy, double dx, double dz) {
  const long total = (long)P * Q;
  const double two_pi = 6.283185307179586476925286766559;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int ky = (int)(i / Q), kx = (int)(i % Q);
    const double kyv = two_pi * freq_index(ky, P) / (P * dy), kxv = two_pi * freq_index(kx, Q) / (Q * dx);
    const double kz = sqrt(fmax(km * km - kyv * kyv - kxv * kxv, 0.0));
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (kz > 0.0) {
      double sn, cs;
      sincos(kz * dz, &sn, &cs);
      const double f = 0.5 * dz / kz;  // -i/2 (cs + i sn) dz / kz = f (sn - i cs)
      v = make_float4((float)cs, (float)sn, (float)(f * sn), (float)(-f * cs));
    }
    EH[i] = v;
  }
}

template <int Q, int MODE>
static cx_status launch_pol_rows(const PolArgs& a, cudaStream_t st) {
  using C = PolRowCfg<Q>;
  auto k = k_pol_rows<Q, MODE>;
  CX_CUDA_TRY(set_smem(k, C::SMEM));
  const long items = (a.N + C::R - 1) / C::R;
  k<<<persistent_grid(k, C::THREADS, C::SMEM, items), C::THREADS, C::SMEM, st>>>(a);
  CX_LAUNCH_CHECK();
  return CX_OK;
}

template <int Q>
static cx_status pol_rows_q(const PolArgs& a, cudaStream_t st) {
  switch (a.mode) {
    case POL_LOAD:
      return launch_pol_rows<Q, POL_LOAD>(a, st);
    case POL_SCATTER:
      return launch_pol_rows<Q, POL_SCATTER>(a, st);
    default:
      return launch_pol_rows<Q, POL_NEXT>(a, st);
  }
}

template <int P, int MODE>
static cx_status launch_pol_cols(const PolArgs& a, cudaStream_t st) {
  using C = PolColCfg<P>;
  auto k = k_pol_cols<P, MODE>;
  CX_CUDA_TRY(set_smem(k, C::SMEM));
  const long items = (a.Q + C::V - 1) / C::V;
  k<<<persistent_grid(k, C::THREADS, C::SMEM, items), C::THREADS, C::SMEM, st>>>(a);
  CX_LAUNCH_CHECK();
  return CX_OK;
}

// padded lengths: even field sizes up to 2048, so 2N is an engine length
#define CX_POL_SIZES(X)                                                                                           \
  X(4) X(6) X(8) X(10) X(12) X(14) X(16) X(20) X(24) X(28) X(32) X(40) X(48) X(56) X(64) X(80) X(96) X(112) X(128) \
  X(160) X(192) X(224) X(256) X(320) X(384) X(448) X(512) X(640) X(768) X(896) X(1024) X(1280) X(1536) X(1792)    \
  X(2048) X(2560) X(3072) X(3584) X(4096)

static cx_status pol_rows(int q, const PolArgs& a, cudaStream_t st) {
  switch (q) {
#define CX_CASE_(N) \
  case N:           \
    return pol_rows_q<N>(a, st);
    CX_POL_SIZES(CX_CASE_)
#undef CX_CASE_
  }
  set_error("padded width %d is not supported", q);
  return CX_ERR_UNSUPPORTED;
}

static cx_status pol_cols(int p, int mode, const PolArgs& a, cudaStream_t st) {
  switch (p) {
#define CX_CASE_(N) \
  case N:           \
    return mode == 1 ? launch_pol_cols<N, 1>(a, st) : launch_pol_cols<N, 2>(a, st);
    CX_POL_SIZES(CX_CASE_)
#undef CX_CASE_
  }
  set_error("padded height %d is not supported", p);
  return CX_ERR_UNSUPPORTED;
}

static bool pol_size_ok(int n) {
  switch (n) {
#define CX_CASE_(N) case N:
    CX_POL_SIZES(CX_CASE_)
#undef CX_CASE_
    return true;
  }
  return false;
}

struct PolPlan {
  size_t off_t1, off_t2, off_w, off_eh, total;
};

static cx_status pol_plan(const cx_polar_desc* d, PolPlan* p) {
  if (!d || d->ny < 2 || d->nx < 2 || d->n_slices < 1 || d->n_wv < 1 || d->wv < 0 || d->wv >= d->n_wv ||
      !(d->wavelength > 0) || !(d->n_medium > 0) || !(d->dy > 0) || !(d->dx > 0)) {
    set_error("invalid polarized multislice descriptor");
    return CX_ERR_INVALID;
  }
  if ((d->ny | d->nx) & 1) {
    set_error("polarized multislice needs even field sizes (the reference pads by N // 2 on each side of the grid "
              "it takes the frequencies from), got %dx%d", d->ny, d->nx);
    return CX_ERR_INVALID;
  }
  if (!pol_size_ok(2 * d->ny) || !pol_size_ok(2 * d->nx)) {
    set_error("padded grid %dx%d: FFT length not supported", 2 * d->ny, 2 * d->nx);
    return CX_ERR_UNSUPPORTED;
  }
  auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
  const size_t P = 2 * (size_t)d->ny, Q = 2 * (size_t)d->nx;
  const size_t tb = al(sizeof(float2) * (size_t)d->ny * Q * 3);
  p->off_t1 = 0;
  p->off_t2 = tb;
  p->off_w = 2 * tb;
  p->off_eh = p->off_w + al(sizeof(float2) * P * Q * 3);
  p->total = p->off_eh + al(sizeof(float4) * P * Q);
  return CX_OK;
}

}  // namespace cx

using namespace cx;

extern "C" cx_status cx_polarized_multislice_workspace_size(const cx_polar_desc* d, size_t* bytes) {
  PolPlan p;
  cx_status s = pol_plan(d, &p);
  if (s != CX_OK) return s;
  if (!bytes) return CX_ERR_INVALID;
  *bytes = p.total;
  return CX_OK;
}

extern "C" cx_status cx_polarized_multislice(const cx_polar_desc* d, const void* u_in, const float* potential,
                                             void* u_out, void* workspace, size_t workspace_bytes,
                                             cx_stream_t stream) {
  PolPlan p;
  cx_status s = pol_plan(d, &p);
  if (s != CX_OK) return s;
  if (!u_in || !potential || !u_out || !workspace) {
    set_error("null pointer argument");
    return CX_ERR_INVALID;
  }
  if (workspace_bytes < p.total) {
    set_error("workspace too small: %zu < %zu", workspace_bytes, p.total);
    return CX_ERR_WORKSPACE;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  char* ws = static_cast<char*>(workspace);
  float2* T1 = reinterpret_cast<float2*>(ws + p.off_t1);
  float2* T2 = reinterpret_cast<float2*>(ws + p.off_t2);
  PolArgs a{};
  a.N = d->ny;
  a.M = d->nx;
  a.P = 2 * d->ny;
  a.Q = 2 * d->nx;
  a.km = 6.283185307179586476925286766559 * d->n_medium / d->wavelength;
  a.NA2km2 = d->NA * d->NA * a.km * a.km;
  a.dy = d->dy;
  a.dx = d->dx;
  a.scale = (float)(1.0 / ((double)a.P * (double)a.Q));
  a.n_wv = d->n_wv;
  a.wv = d->wv;
  a.u_in = static_cast<const float2*>(u_in);
  a.u_out = static_cast<float2*>(u_out);
  a.V = potential;
  a.W = reinterpret_cast<float2*>(ws + p.off_w);
  a.EH = reinterpret_cast<const float4*>(ws + p.off_eh);
  if ((s = ensure_twiddles(&a.twg)) != CX_OK) return s;
  {
    long total = (long)a.P * a.Q, g = (total + 255) / 256;
    if (g > (long)sm_count() * 16) g = (long)sm_count() * 16;
    k_pol_table<<<(int)g, 256, 0, st>>>(reinterpret_cast<float4*>(ws + p.off_eh), a.P, a.Q, a.km, d->dy, d->dx,
                                        d->dz);
    CX_LAUNCH_CHECK();
  }
  // T1 = FFT_x(pad u)
  a.mode = POL_LOAD;
  a.Tout = T1;
  if ((s = pol_rows(a.Q, a, st)) != CX_OK) return s;
  for (int i = 0; i < d->n_slices; ++i) {
    a.slice = i;
    a.Tin = T1;  // C1: T2 = IFFT_y(Q U) rows < N, W = e U
    a.Tout = T2;
    if ((s = pol_cols(a.P, 1, a, st)) != CX_OK) return s;
    a.mode = POL_SCATTER;  // R2: T1 = FFT_x(pad(V_i a)), a = crop IFFT_x(T2) / (P Q)
    a.Tin = T2;
    a.Tout = T1;
    if ((s = pol_rows(a.Q, a, st)) != CX_OK) return s;
    a.Tin = T1;  // C2: T2 = IFFT_y(Q (W + h S)) rows < N
    a.Tout = T2;
    if ((s = pol_cols(a.P, 2, a, st)) != CX_OK) return s;
    a.mode = POL_NEXT;  // R3: u = crop IFFT_x(T2) / (P Q); T1 = FFT_x(pad u) unless last
    a.last = i + 1 == d->n_slices;
    a.Tin = T2;
    a.Tout = T1;
    if ((s = pol_rows(a.Q, a, st)) != CX_OK) return s;
    a.last = 0;
  }
  return CX_OK;
}
