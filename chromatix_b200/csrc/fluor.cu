// Fluorescent thick sample (functional/samples.py:285-441): Monte-Carlo
// samples of random fluorophore phases; per sample a forward multislice with
// the fluorescence added before every slice propagation, then the backward
// stack of intensities |crop(IFFT2(U H_b^(i+1)))|^2, U = FFT2(u_D).
//
// Forward (multislice row / column passes, state = FFT_x(u) / px between a
// column and a row pass):
//   load u_0 / px -> for i < D: row pass IFFT_x, v exp(i k dz dn_i) + fl_i exp(i ph_i), FFT_x;
//                               column pass FFT_y x H(dz) IFFT_y
// Backward: H_b^(i+1) = H(-(i+1) dz) with the band limit of dz (|z| and a
// conjugate phase for z < 0, as compute_asm_propagator; the limit and the
// evanescent mask are powers of themselves), so plane i of the stack is the
// column FFT of the forward state (once per sample), times H(-(i+1) dz), the
// column inverse and the prop2d inverse row pass; the planes are cropped in
// those passes and summed as px^2 |.|^2 / S into out[D - 1 - i].
// The reference carries the field from one sample into the next: sample s + 1
// starts from U_s H_b^D (a spectrum, used as a field): px U H(-D dz), an
// elementwise product with the spectrum U = FFT_y(state) that the backward
// planes share (k_fluor_cols computes it once per sample).
#include <cmath>
#include <cstdint>
#include <type_traits>
#include <vector>

#include "multislice.cuh"

namespace cx {

// counter-based phases: splitmix64 of seed + (c + 1) * golden gamma, top 24
// bits as u in [0, 1), phase = float(2 pi) * u; c = s * D ny nx + index
__global__ void k_fluor_phases(float* __restrict__ ph, long n, uint64_t seed, uint64_t c0) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    uint64_t z = seed + (c0 + (uint64_t)i + 1ull) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    const float u = (float)(uint32_t)(z >> 40) * (1.0f / 16777216.0f);
    ph[i] = 6.28318530717958647692f * u;
  }
}

// out[D - 1 - (c0 + q)] += w |O[q]|^2 for the nb planes of a chunk
__global__ void k_fluor_accumulate(const float2* __restrict__ O, float* __restrict__ out, int c0, int nb, int D,
                                   long plane, float w) {
  const long total = (long)nb * plane;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int q = (int)(i / plane);
    const long r = i - (long)q * plane;
    const float2 v = O[i];
    out[(size_t)(D - 1 - (c0 + q)) * plane + r] += w * (v.x * v.x + v.y * v.y);
  }
}

__global__ void k_fluor_fill_h(float2* __restrict__ H, Prop2DArgs a, const cx_plane* pl) {
  const long total = (long)a.py * a.px;
  const cx_plane p = *pl;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x)
    H[i] = prop_kernel(i / a.px, i % a.px, a, p);
}

// Column passes of the backward stack, V-column tiles as k_prop_cols:
//   FLUOR_SPEC: U = FFT_y(S) of the forward state, all rows (once per sample)
//   FLUOR_BACK: plane q of a chunk: IFFT_y(U H(z_q)) / (py px), rows
//               [pad, pad + ny) into T2 (q, ny, px) -- the column pass of
//               k_prop_cols without its forward transform, which is the same
//               for every plane
//   FLUOR_FWD:  the forward slice step, FFT_y x H(dz) (table) IFFT_y / (py px), in place
enum FluorCol { FLUOR_SPEC = 0, FLUOR_BACK = 1, FLUOR_FWD = 2 };

// Narrow column tiles for the single-plane forward pass: at least 4 columns
// (32-byte row segments), whole warps for exact-size teams, at most the
// column configuration's width.  At 384^2 the column configuration's
// 16-column tiles give 24 CTAs; 4-column tiles give 96.
template <int N>
struct NarrowColCfg {
  using C0 = ColCfg<N>;
  static constexpr bool CTA = C0::CTA;
  static constexpr int LPV = C0::LPV;
  static constexpr int pick() {
    int v = 4;
    while (CTA && (v * LPV) % 32 != 0) v *= 2;
    return v < C0::V ? v : C0::V;
  }
  static constexpr int V = pick();
  static_assert(!CTA || (V * LPV) % 32 == 0, "exact-size teams must fill whole warps");
  static constexpr int LEN = col_len(N, V);
  static constexpr int THREADS = V * LPV;
  static constexpr int TW = tw_len(N);
  static constexpr int MINB = minb_for(THREADS);
  static constexpr size_t SMEM = sizeof(float2) * ((size_t)TW + (size_t)V * LEN);
};

template <int NY, int MODE>
using FluorColCfg = typename std::conditional<MODE == FLUOR_FWD, NarrowColCfg<NY>, ColCfg<NY>>::type;

// no blocks-per-SM bound: the FP64 propagator in the staged load needs
// about 90 registers, more than the column configuration's bound leaves
// Base ASM propagator of |z| = dz per frequency (FFT order), FP64: {v, kind}
// with kind 1 propagating (phase v = K sqrt(kern)), 2 evanescent (decay
// v = K sqrt(-kern)), 0 outside the band limit -- the FP64 branch of
// prop_kernel_accurate with shift 0.  Plane z = -m dz then has phase -m v
// (the conjugate) or decay exp(-m v), m = |z| / dz: the multiplier is
// linear in |z|, so the square root and the divisions run once per call.
__global__ void k_fluor_ptable(double2* __restrict__ tab, Prop2DArgs a, const cx_plane* plp) {
  const cx_plane pl = *plp;
  const double K = 6.283185307179586476925286766559 * fabs(pl.z) * a.n_med / pl.wavelength;
  const double q = pl.wavelength / a.n_med;
  const long total = (long)a.py * a.px;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int ky = (int)(i / a.px), kx = (int)(i % a.px);
    const double fy = (double)freq_index(ky, a.py) / ((double)a.py * pl.dy);
    const double fx = (double)freq_index(kx, a.px) / ((double)a.px * pl.dx);
    double2 e = make_double2(0.0, 0.0);
    if (!(a.bandlimit && (fabs(fy - pl.bl_y0) > pl.bl_hy || fabs(fx - pl.bl_x0) > pl.bl_hx))) {
      const double gy = fy - a.ky0, gx = fx - a.kx0;
      const double kern = 1.0 - q * q * (gy * gy + gx * gx);
      if (kern >= 0.0 || a.remove_evanescent)
        e = make_double2(K * sqrt(kern > 0.0 ? kern : 0.0), 1.0);
      else
        e = make_double2(K * sqrt(-kern), 2.0);
    }
    tab[i] = e;
  }
}

template <int NY, int MODE>
__global__ void __launch_bounds__(FluorColCfg<NY, MODE>::THREADS, 1)
    k_fluor_cols(const float2* T, float2* T2, Prop2DArgs a, int nb, const double2* __restrict__ tab,
                 double inv_dz) {
  using C = FluorColCfg<NY, MODE>;
  constexpr int V = C::V, LEN = C::LEN;
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* tile = sm + C::TW;
  load_twiddles<NY>(tw, a.twg, threadIdx.x, blockDim.x);
  const int team = threadIdx.x / C::LPV, lane = threadIdx.x % C::LPV;
  float2* s = tile + team * LEN;
  const int tiles_x = (a.px + V - 1) / V;
  const long total = (long)tiles_x * (MODE == FLUOR_BACK ? nb : 1);
  const float scale = 1.0f / ((float)a.py * (float)a.px);
  for (long t = blockIdx.x; t < total; t += gridDim.x) {
    const int q = (int)(t / tiles_x);
    const int x0 = (int)(t % tiles_x) * V;
    __syncthreads();
    load_col_tile<V, LEN>(tile, T, a.px, x0, a.px, 0, a.py, [](int r) { return r; });
    __syncthreads();
    const int kx = x0 + team;
    const bool valid = kx < a.px;
    auto load1 = [&](int n) -> float2 { return s[pad_idx(n)]; };
    if constexpr (MODE == FLUOR_SPEC) {
      auto store1 = [&](int k, float2 v, int) { s[pad_idx(k)] = v; };
      team_fft<NY, false, C::LPV, C::CTA>(s, tw, lane, team, load1, store1);
    } else if constexpr (MODE == FLUOR_FWD) {
      // H(dz) from the explicit table (a.H, FFT order)
      auto store1 = [&](int k, float2 v, int) { s[pad_idx(k)] = valid ? cmul(v, a.H[(size_t)k * a.px + kx]) : v; };
      team_fft<NY, false, C::LPV, C::CTA>(s, tw, lane, team, load1, store1);
      team_barrier<C::LPV, C::CTA>(team);
      auto load2 = [&](int n) -> float2 { return s[pad_idx(n)]; };
      auto store2 = [&](int k, float2 v, int) { s[pad_idx(k)] = cscale(v, scale); };
      team_fft<NY, true, C::LPV, C::CTA>(s, tw, lane, team, load2, store2);
    } else {
      const cx_plane pl = a.planes[q];
      const double m = rint(fabs(pl.z) * inv_dz);  // the plane's multiple of dz
      const bool neg = pl.z < 0.0;
      auto loadh = [&](int n) -> float2 {
        const float2 v = s[pad_idx(n)];
        if (!valid) return v;
        const double2 e = tab[(size_t)n * a.px + kx];
        float2 h = make_float2(0.f, 0.f);
        if (e.y == 1.0) {
          h = expi_reduced(neg ? -m * e.x : m * e.x);
        } else if (e.y == 2.0) {
          h = make_float2(expf((float)(-m * e.x)), 0.f);
        }
        return cscale(cmul(v, h), scale);
      };
      auto store1 = [&](int k, float2 v, int) { s[pad_idx(k)] = v; };
      team_fft_ex<NY, true, true, false, C::LPV, C::CTA>(s, tw, lane, team, loadh, store1);
    }
    __syncthreads();
    const int r0 = MODE == FLUOR_BACK ? a.out_y0 : 0;
    const int nr = MODE == FLUOR_BACK ? a.out_ny : a.py;
    for (int idx = threadIdx.x; idx < nr * V; idx += blockDim.x) {
      const int r = idx / V, c = idx % V, x = x0 + c;
      if (x < a.px) T2[((size_t)q * nr + r) * a.px + x] = tile[c * LEN + pad_idx(r0 + r)];
    }
  }
}

template <int NY, int MODE>
static cx_status launch_fluor_cols(const float2* T, float2* T2, const Prop2DArgs& a, int nb, const double2* tab,
                                   double inv_dz, cudaStream_t st) {
  using C = FluorColCfg<NY, MODE>;
  auto k = k_fluor_cols<NY, MODE>;
  CX_CUDA_TRY(set_smem(k, C::SMEM));
  const long units = (long)((a.px + C::V - 1) / C::V) * (MODE == FLUOR_BACK ? nb : 1);
  k<<<persistent_grid(k, C::THREADS, C::SMEM, units), C::THREADS, C::SMEM, st>>>(T, T2, a, nb, tab, inv_dz);
  CX_LAUNCH_CHECK();
  return CX_OK;
}

static cx_status dispatch_fluor_cols(int n, int mode, const float2* T, float2* T2, const Prop2DArgs& a, int nb,
                                     const double2* tab, double inv_dz, cudaStream_t st) {
  switch (n) {
#define CX_CASE_(N)                                                                              \
  case N:                                                                                        \
    return mode == FLUOR_SPEC  ? launch_fluor_cols<N, FLUOR_SPEC>(T, T2, a, nb, tab, inv_dz, st) \
           : mode == FLUOR_FWD ? launch_fluor_cols<N, FLUOR_FWD>(T, T2, a, nb, tab, inv_dz, st)  \
                               : launch_fluor_cols<N, FLUOR_BACK>(T, T2, a, nb, tab, inv_dz, st);
    CX_FOR_EACH_SIZE(CX_CASE_)
#undef CX_CASE_
  }
  set_error("FFT length %d is not supported", n);
  return CX_ERR_UNSUPPORTED;
}

// the carry, in place: V = scale U H(z) (an elementwise product with the spectrum)
__global__ void k_fluor_carry(float2* __restrict__ U, Prop2DArgs a, const cx_plane* pl, float scale) {
  const long total = (long)a.py * a.px;
  const cx_plane p = *pl;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x)
    U[i] = cscale(cmul(U[i], prop_kernel((int)(i / a.px), (int)(i % a.px), a, p)), scale);
}

static constexpr int kFluorChunk = 32;  // backward planes per column / row pass

struct FluorPlan {
  int py, px, D, S, CH;
  Prop2DArgs col;
  size_t off_h, off_f, off_v, off_ph, off_t2, off_o, off_tab, total;
};

static size_t fal(size_t b) { return (b + 255) & ~(size_t)255; }

static cx_status fluor_plan(const cx_fluor_desc* d, FluorPlan* p) {
  if (!d || d->ny <= 0 || d->nx <= 0 || d->pad < 0 || d->n_slices <= 0 || d->num_samples <= 0 ||
      !(d->wavelength > 0.0) || !(d->dy > 0.0) || !(d->dx > 0.0) || !(d->n_medium > 0.0)) {
    set_error("invalid fluorescent multislice descriptor");
    return CX_ERR_INVALID;
  }
  p->py = d->ny + 2 * d->pad;
  p->px = d->nx + 2 * d->pad;
  if (!size_supported(p->py) || !size_supported(p->px)) {
    set_error("padded grid %dx%d: FFT length not supported", p->py, p->px);
    return CX_ERR_UNSUPPORTED;
  }
  p->D = d->n_slices;
  p->S = d->num_samples;
  p->CH = p->D < kFluorChunk ? p->D : kFluorChunk;
  Prop2DArgs& a = p->col;
  a.ny = p->py;
  a.nx = p->px;
  a.py = p->py;
  a.px = p->px;
  a.pad_y = 0;
  a.pad_x = 0;
  a.W = 1;
  a.n_in_planes = 1;
  a.n_out_planes = 1;
  a.out_y0 = 0;
  a.out_ny = p->py;
  a.out_x0 = 0;
  a.out_nx = p->px;
  a.kernel = CX_KERNEL_ASM;
  a.precision = CX_PREC_ACCURATE;
  a.remove_evanescent = d->remove_evanescent;
  a.bandlimit = d->bandlimit;
  a.n_med = d->n_medium;
  a.ky0 = d->ky0;
  a.kx0 = d->kx0;
  a.na_f2 = -1.0;
  a.precise = 0;
  a.conj_h = 0;
  a.planes = nullptr;
  a.H = nullptr;
  const size_t field = sizeof(float2) * (size_t)p->py * p->px;
  p->off_h = fal(sizeof(cx_plane) * (size_t)(p->D + 2));
  p->off_f = p->off_h + fal(field);
  p->off_v = p->off_f + fal(field);
  p->off_ph = p->off_v + fal(field);
  p->off_t2 = p->off_ph + fal(sizeof(float) * (size_t)p->D * d->ny * d->nx);
  p->off_o = p->off_t2 + fal(sizeof(float2) * (size_t)p->CH * d->ny * p->px);
  p->off_tab = p->off_o + fal(sizeof(float2) * (size_t)p->CH * d->ny * d->nx);
  p->total = p->off_tab + fal(sizeof(double2) * (size_t)p->py * p->px);
  return ensure_twiddles(&a.twg);
}

// planes: 0 the slice (+dz), 1 + i the backward plane -(i + 1) dz, D + 1 the
// carry -D dz; every one with the band limit of |z| = dz
static cx_status fluor_upload_planes(const cx_fluor_desc* d, const FluorPlan& p, cx_plane* dev, cx_plane* host,
                                     cudaStream_t st) {
  double bl[4] = {0, 0, 0, 0};
  if (d->bandlimit) {
    // Matsushima band limit for |z| = dz, shift 0 (propagation.py:557-579)
    const double ext[2] = {d->dy * p.py, d->dx * p.px};
    for (int i = 0; i < 2; ++i) {
      const double df = 1.0 / ext[i];
      const double klp = std::pow(std::pow(1.0 / (2 * df), -2.0) * d->dz * d->dz + 1.0, -0.5) / d->wavelength;
      const double kln = std::pow(std::pow(-1.0 / (2 * df), -2.0) * d->dz * d->dz + 1.0, -0.5) / d->wavelength;
      bl[i] = 0.5 * (klp - kln);
      bl[2 + i] = 0.5 * (klp + kln);
    }
  }
  for (int i = 0; i < p.D + 2; ++i) {
    cx_plane& q = host[i];
    q = cx_plane{};
    q.z = i == 0 ? d->dz : -(double)(i <= p.D ? i : p.D) * d->dz;
    q.wavelength = d->wavelength;
    q.dy = d->dy;
    q.dx = d->dx;
    q.bl_y0 = bl[0];
    q.bl_x0 = bl[1];
    q.bl_hy = bl[2];
    q.bl_hx = bl[3];
  }
  CX_CUDA_TRY(cudaMemcpyAsync(dev, host, sizeof(cx_plane) * (size_t)(p.D + 2), cudaMemcpyHostToDevice, st));
  return CX_OK;
}

static int grid_for(long n) {
  long g = (n + 255) / 256;
  const long cap = (long)sm_count() * 16;
  return (int)(g < 1 ? 1 : (g > cap ? cap : g));
}

}  // namespace cx

using namespace cx;

extern "C" cx_status cx_fluorescent_multislice_workspace_size(const cx_fluor_desc* d, size_t* bytes) {
  FluorPlan p;
  cx_status s = fluor_plan(d, &p);
  if (s != CX_OK) return s;
  if (!bytes) return CX_ERR_INVALID;
  *bytes = p.total;
  return CX_OK;
}

extern "C" cx_status cx_fluorescent_multislice(const cx_fluor_desc* d, const void* u_in, const float* fluorescence,
                                               const float* dn, const float* phases, float* out, void* workspace,
                                               size_t workspace_bytes, cx_stream_t stream) {
  FluorPlan p;
  cx_status s = fluor_plan(d, &p);
  if (s != CX_OK) return s;
  if (!u_in || !fluorescence || !dn || !out || !workspace) {
    set_error("null pointer argument");
    return CX_ERR_INVALID;
  }
  if (workspace_bytes < p.total) {
    set_error("workspace too small: %zu < %zu", workspace_bytes, p.total);
    return CX_ERR_WORKSPACE;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  char* w = static_cast<char*>(workspace);
  cx_plane* planes = reinterpret_cast<cx_plane*>(w);
  float2* Hf = reinterpret_cast<float2*>(w + p.off_h);
  float2* F = reinterpret_cast<float2*>(w + p.off_f);
  float2* V = reinterpret_cast<float2*>(w + p.off_v);
  float* ph_buf = reinterpret_cast<float*>(w + p.off_ph);
  float2* T2 = reinterpret_cast<float2*>(w + p.off_t2);
  float2* O = reinterpret_cast<float2*>(w + p.off_o);
  double2* tab = reinterpret_cast<double2*>(w + p.off_tab);
  std::vector<cx_plane> host(p.D + 2);
  if ((s = fluor_upload_planes(d, p, planes, host.data(), st)) != CX_OK) return s;
  // the slice propagator table H(dz), FP64 sin / cos
  {
    Prop2DArgs a = p.col;
    a.precise = 1;
    k_fluor_fill_h<<<grid_for((long)p.py * p.px), 256, 0, st>>>(Hf, a, planes);
    CX_LAUNCH_CHECK();
    k_fluor_ptable<<<grid_for((long)p.py * p.px), 256, 0, st>>>(tab, p.col, planes);
    CX_LAUNCH_CHECK();
  }
  // plane multiples of |dz| (dz = 0: every plane's propagator is 1, m = 0)
  const double inv_dz = d->dz != 0.0 ? 1.0 / std::fabs(d->dz) : 0.0;
  const long plane = (long)d->ny * d->nx;
  const long stack = plane * p.D;
  CX_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(float) * (size_t)stack, st));

  MsArgs m{};
  m.ny = d->ny;
  m.nx = d->nx;
  m.pad_y = d->pad;
  m.pad_x = d->pad;
  m.py = p.py;
  m.px = p.px;
  m.precision = CX_PREC_ACCURATE;
  m.lam = d->wavelength;
  m.dz = d->dz;
  m.kdz_f = (float)(6.283185307179586476925286766559 * d->dz / d->wavelength);
  m.twg = p.col.twg;
  m.dn = dn;
  m.fl = fluorescence;
  m.buf = F;
  m.record = 0;
  const float w_sample = (float)((double)p.px * (double)p.px / (double)p.S);
  for (int smp = 0; smp < p.S; ++smp) {
    // u_0: the padded input field (sample 0) or the carry of the previous sample
    m.mode = MS_LOAD;
    m.load_scale = 1.0f / (float)p.px;
    if (smp == 0) {
      m.src = static_cast<const float2*>(u_in);
      m.sy = d->ny;
      m.sx = d->nx;
      m.oy = d->pad;
      m.ox = d->pad;
    } else {
      m.src = V;
      m.sy = p.py;
      m.sx = p.px;
      m.oy = 0;
      m.ox = 0;
    }
    if ((s = ms_dispatch_rows(p.px, m, st)) != CX_OK) return s;
    if (phases) {
      m.ph = phases + (size_t)smp * stack;
    } else {
      k_fluor_phases<<<grid_for(stack), 256, 0, st>>>(ph_buf, stack, d->seed, (uint64_t)smp * (uint64_t)stack);
      CX_LAUNCH_CHECK();
      m.ph = ph_buf;
    }
    m.mode = MS_FLUOR;
    for (int i = 0; i < p.D; ++i) {
      m.slice = i;
      if ((s = ms_dispatch_rows(p.px, m, st)) != CX_OK) return s;
      Prop2DArgs a = p.col;
      a.planes = planes;
      a.kernel = CX_KERNEL_EXPLICIT;
      a.H = Hf;
      if ((s = dispatch_fluor_cols(p.py, FLUOR_FWD, F, F, a, 1, tab, inv_dz, st)) != CX_OK) return s;
    }
    // U = FFT_y(state) once, into V; then the backward planes, cropped, in chunks of CH
    if ((s = dispatch_fluor_cols(p.py, FLUOR_SPEC, F, V, p.col, 1, tab, inv_dz, st)) != CX_OK) return s;
    for (int c0 = 0; c0 < p.D; c0 += p.CH) {
      const int nb = p.D - c0 < p.CH ? p.D - c0 : p.CH;
      Prop2DArgs b = p.col;
      b.planes = planes + 1 + c0;
      b.n_out_planes = nb;
      b.out_y0 = d->pad;
      b.out_ny = d->ny;
      b.out_x0 = d->pad;
      b.out_nx = d->nx;
      if ((s = dispatch_fluor_cols(p.py, FLUOR_BACK, V, T2, b, nb, tab, inv_dz, st)) != CX_OK) return s;
      if ((s = dispatch_rows_inv(p.px, T2, O, b, st)) != CX_OK) return s;
      k_fluor_accumulate<<<grid_for((long)nb * plane), 256, 0, st>>>(O, out, c0, nb, p.D, plane, w_sample);
      CX_LAUNCH_CHECK();
    }
    if (smp + 1 < p.S) {
      // carry: U H_b^D = px FFT_y(state) H(-D dz), a spectrum in field layout (in place in V)
      k_fluor_carry<<<grid_for((long)p.py * p.px), 256, 0, st>>>(V, p.col, planes + p.D + 1, (float)p.px);
      CX_LAUNCH_CHECK();
    }
  }
  return CX_OK;
}
