// Batched 4f widefield PSF, fused end to end.
//
// Reference composition (systems/microscopes.py:334-355, README.md:55-85):
//   objective_point_source   functional/sources.py:122-209
//   phase_change             functional/phase_masks.py:29-68, 105-124
//   ff_lens                  functional/lenses.py:64-95
//     optical_fft            functional/convenience.py:9-59  (fftshift(fft2(ifftshift(.))))
//   Field.intensity          core/field.py:735-740
//
// pass 0  count the pupil pixels per wavelength (the source's power
//         normalisation: |u|^2 is amp^2 / L^4 on every pupil pixel)
// pass A  per (z, wavelength, row): evaluate source * pupil * mask * lens
//         normalisation in the FFT loader (ifftshift = index remap), FFT
//         along x, write the row spectrum (rows outside the pupil are
//         skipped: their spectrum is zero)
// pass B  per (z, V-column tile): for every wavelength FFT along y and add
//         density * |X|^2 into per-lane registers; store the fftshifted
//         intensity once.
// The z axis is processed in chunks so the row spectra of a chunk stay in L2
// between pass A and pass B.
#pragma once
#include "host.cuh"

namespace cx {

constexpr int PSF_MAX_WV = 8;

struct PsfWv {
  double lam, dens, dy, dx;
  double L2;       // lam f / n  (L^2 of the source, sources.py:201)
  double R2;       // source pupil radius^2 ((lam0/lam) D/2)^2 (pupils.py:19-22)
  double RL2;      // lens pupil radius^2 (or < 0: none)
  double mod;      // lam0 / lam (spectral modulation of the mask)
  double lens_re, lens_im;  // optical_fft normalisation -1j dy dx / L_sq
  float L2f, R2f, RL2f, modf;  // float32 versions for the reference-order mode
};

struct PsfArgs {
  int ny, nx, nz, W, precision, has_phase, normalize;
  int z0, zc;  // chunk start and length
  double f_obj, n, amp, offy, offx, power;
  PsfWv wv[PSF_MAX_WV];
  int ylo[PSF_MAX_WV], nrows[PSF_MAX_WV], prefix[PSF_MAX_WV], rowsum;  // compact row spectra
  // accurate mode: the source is evaluated from tables built once per call.
  // M (z-independent, per wavelength w a box of nrows_w x ncols_w pixels from
  // (ylo_w, xlo_w)): amp (-1j / L^2) sqrt(P / power) lens_norm exp(i phase mod)
  // on pupil pixels, 0 elsewhere.  CX (nz, csum): exp(i qz (x dx - off_x)^2),
  // qz = -pi (z / f) / L^2.  The defocus phase is separable, so a pixel is
  // M(y, x) CX(z, x) exp(i qz (y dy - off_y)^2).
  int xlo[PSF_MAX_WV], ncols[PSF_MAX_WV], mprefix[PSF_MAX_WV], cprefix[PSF_MAX_WV];
  long msum;
  int csum;
  float2* M;
  float2* CX;
  const double* z;
  const float* phase;
  float2* T;  // (zc, rowsum, nx): only the rows [ylo_w, ylo_w + nrows_w) of each wavelength
  const unsigned long long* counts;  // [0, 8): pupil pixel counts per wavelength
  const int* srange;                 // [0, 8): ny - first support row ; [8, 16): last support row + 1
  float* out;
  const float2* twg;  // device twiddle tables (ensure_twiddles)
};

// exact pupil row range [first, last + 1) of wavelength w (from the count pass)
__device__ __forceinline__ int support_lo(const PsfArgs& a, int w) { return a.ny - a.srange[w]; }
__device__ __forceinline__ int support_hi(const PsfArgs& a, int w) { return a.srange[8 + w]; }

// support predicate shared by all passes (accurate: FP64, ref32: float32)
__device__ __forceinline__ bool in_pupil(const PsfArgs& a, const PsfWv& p, int y, int x) {
  if (a.precision == CX_PREC_REF32) {
    const float gy = fm((float)p.dy, (float)y - (float)a.ny * 0.5f);
    const float gx = fm((float)p.dx, (float)x - (float)a.nx * 0.5f);
    const float r2 = fa(fm(gy, gy), fm(gx, gx));
    return r2 <= p.R2f && (p.RL2f < 0.f || r2 <= p.RL2f);
  }
  const double gy = p.dy * ((double)y - (double)a.ny * 0.5);
  const double gx = p.dx * ((double)x - (double)a.nx * 0.5);
  const double r2 = gy * gy + gx * gx;
  return r2 <= p.R2 && (p.RL2 < 0.0 || r2 <= p.RL2);
}

__device__ __forceinline__ bool row_has_support(const PsfArgs& a, const PsfWv& p, int y) {
  if (a.precision == CX_PREC_REF32) {
    const float gy = fm((float)p.dy, (float)y - (float)a.ny * 0.5f);
    const float r2 = fm(gy, gy);
    return r2 <= p.R2f && (p.RL2f < 0.f || r2 <= p.RL2f);
  }
  const double gy = p.dy * ((double)y - (double)a.ny * 0.5);
  const double r2 = gy * gy;
  return r2 <= p.R2 && (p.RL2 < 0.0 || r2 <= p.RL2);
}

// per-wavelength complex constant of the fused source (everything but the
// per-pixel phase): amp * (-1j / L^2) * sqrt(P / power_w) * lens_norm
__device__ __forceinline__ float2 psf_const(const PsfArgs& a, int w, const unsigned long long* counts) {
  double scale = 1.0;
  if (a.normalize) {
    // Field.power of a chromatic field (core/field.py:728-733):
    // area_w * sum_w' density_w' * sum_yx |u_w'|^2
    double s = 0.0;
    for (int v = 0; v < a.W; ++v) s += a.wv[v].dens * (a.amp * a.amp) / (a.wv[v].L2 * a.wv[v].L2) * (double)counts[v];
    const double pw = a.wv[w].dy * a.wv[w].dx * s;
    scale = pw > 0.0 ? sqrt(a.power / pw) : 0.0;
  }
  // (-1j / L^2) * amp * scale  times lens normalisation (lens_re + i lens_im)
  const double sre = 0.0, sim = -a.amp * scale / a.wv[w].L2;
  const double re = sre * a.wv[w].lens_re - sim * a.wv[w].lens_im;
  const double im = sre * a.wv[w].lens_im + sim * a.wv[w].lens_re;
  return make_float2((float)re, (float)im);
}

// ---------------------------------------------------------------------------
// pass A: analytic source -> row FFT, for the rows inside the pupil only
// ---------------------------------------------------------------------------
// accurate mode: the loader is M * CX * one FP64 row factor (see PsfArgs).
// Every team runs one transform per iteration (rows past the end or outside
// the pupil transform zeros and store nothing), so teams can have the exact
// lane count and share CTA-wide barriers.
template <int NX>
using PsfRowCfg = RowCfgX<NX>;

template <int NX, int Q>
__global__ void __launch_bounds__(PsfRowCfg<NX>::THREADS, PsfRowCfg<NX>::MINB) k_psf_rows_tab(PsfArgs a) {
  using C = PsfRowCfg<NX>;
  extern __shared__ float2 sm[];
  float2* tw = sm;
  load_twiddles<NX>(tw, a.twg, threadIdx.x, blockDim.x);
  __syncthreads();
  const int team = threadIdx.x / C::LPV, lane = threadIdx.x % C::LPV;
  float2* s = sm + C::TW + team * Plan<NX>::LEN;
  const long total = (long)a.zc * a.rowsum;
  const double PI = 3.141592653589793238462643383279502884;
  for (long base = (long)blockIdx.x * C::TEAMS; base < total; base += (long)gridDim.x * C::TEAMS) {
    const long item0 = base + team;
    const long item = item0 < total ? item0 : total - 1;
    const int zl = (int)(item / a.rowsum);
    const int rem = (int)(item % a.rowsum);
    int w = 0;
    while (w + 1 < a.W && rem >= a.prefix[w + 1]) ++w;
    const PsfWv& p = a.wv[w];
    const int y = a.ylo[w] + (rem - a.prefix[w]);
    const bool live = item0 < total && y >= support_lo(a, w) && y < support_hi(a, w);
    const double z = a.z[a.z0 + zl];
    const double gyo = p.dy * ((double)y - (double)a.ny * 0.5) - a.offy;
    const double qz = -PI * (z / a.f_obj) / p.L2;
    const float2* mrow = a.M + a.mprefix[w] + (size_t)(y - a.ylo[w]) * a.ncols[w];
    const float2* cxz = a.CX + (size_t)(a.z0 + zl) * a.csum + a.cprefix[w];
    const int xlo = a.xlo[w], nc = live ? a.ncols[w] : 0;
    const float2 cy = expi_precise(qz * gyo * gyo);
    float2* dst = a.T + ((size_t)zl * a.rowsum + rem) * a.nx;
    auto load = [&](int n) -> float2 {
      const int c = add_mod(n, NX / 2, NX) - xlo;  // ifftshift along x, then the box column
      if ((unsigned)c >= (unsigned)nc) return make_float2(0.f, 0.f);
      return cmul(cmul(mrow[c], cxz[c]), cy);
    };
    auto store = [&](int k, float2 v, int) {
      if (live) dst[k] = v;
    };
    team_fft<NX, false, C::LPV, C::CTA, (Q > 0 ? edge_zero_mask<NX, Q>() : 0u)>(s, tw, lane, team, load, store);
  }
}

// reference-order float32 mode: the source evaluated per pixel in the loader
template <int NX>
__global__ void __launch_bounds__(RowCfg<NX>::THREADS, RowCfg<NX>::MINB) k_psf_rows(PsfArgs a) {
  using C = RowCfg<NX>;
  extern __shared__ float2 sm[];
  float2* tw = sm;
  __shared__ float2 cw[PSF_MAX_WV];
  load_twiddles<NX>(tw, a.twg, threadIdx.x, blockDim.x);
  if (threadIdx.x < a.W) cw[threadIdx.x] = psf_const(a, threadIdx.x, a.counts);
  __syncthreads();
  const int team = threadIdx.x / C::LPV, lane = threadIdx.x % C::LPV;
  float2* s = sm + C::TW + team * Plan<NX>::LEN;
  const long total = (long)a.zc * a.rowsum;
  const double PI = 3.141592653589793238462643383279502884;
  for (long base = (long)blockIdx.x * C::TEAMS; base < total; base += (long)gridDim.x * C::TEAMS) {
    const long item = base + team;
    if (item >= total) continue;
    const int zl = (int)(item / a.rowsum);
    const int rem = (int)(item % a.rowsum);
    int w = 0;
    while (w + 1 < a.W && rem >= a.prefix[w + 1]) ++w;
    const PsfWv& p = a.wv[w];
    const int y = a.ylo[w] + (rem - a.prefix[w]);
    // rows outside the pupil have a zero spectrum: the whole team skips them
    // (team barriers are team-local, so teams sharing a warp may diverge)
    if (y < support_lo(a, w) || y >= support_hi(a, w)) continue;
    const double z = a.z[a.z0 + zl];
    const float2 cst = cw[w];
    const float* ph_row = a.has_phase ? a.phase + (size_t)y * a.nx : nullptr;
    const double gy = p.dy * ((double)y - (double)a.ny * 0.5);
    const double qz = -PI * (z / a.f_obj) / p.L2;
    const double gyo = gy - a.offy;
    float2* dst = a.T + ((size_t)zl * a.rowsum + rem) * a.nx;
    auto store = [&](int k, float2 v, int) { dst[k] = v; };
    auto load = [&](int n) -> float2 {
      const int x = add_mod(n, NX / 2, NX);  // ifftshift along x
      if (!in_pupil(a, p, y, x)) return make_float2(0.f, 0.f);
      if (a.precision == CX_PREC_REF32) {
        // objective_point_source: u = (amp*-1j/L^2) * exp(1j*phase) (sources.py:201-204)
        const float gyf = fm((float)p.dy, (float)y - (float)a.ny * 0.5f);
        const float gxf = fm((float)p.dx, (float)x - (float)a.nx * 0.5f);
        const float dyo = fs(gyf, (float)a.offy), dxo = fs(gxf, (float)a.offx);
        const float r2 = fa(fm(dyo, dyo), fm(dxo, dxo));
        const float phs = fd(fm(fm(-3.14159265358979f, fd((float)z, (float)a.f_obj)), r2), p.L2f);
        float s1, c1;
        sincosf(phs, &s1, &c1);
        float2 v = cmul(cst, make_float2(c1, s1));
        if (a.has_phase) {
          float s2, c2;
          sincosf(fm(ph_row[x], p.modf), &s2, &c2);
          v = cmul(v, make_float2(c2, s2));
        }
        return v;
      }
      const double gxo = p.dx * ((double)x - (double)a.nx * 0.5) - a.offx;
      double ph = qz * (gyo * gyo + gxo * gxo);
      if (a.has_phase) ph += (double)ph_row[x] * p.mod;
      return cmul(cst, expi_reduced(ph));
    };
    team_fft_ex<NX, false, true, false>(s, tw, lane, team, load, store);
  }
}

// ---------------------------------------------------------------------------
// pass B: column FFTs of every wavelength, spectral intensity sum (kept in a
// shared accumulator), fftshifted coalesced store
// ---------------------------------------------------------------------------
template <int NY>
struct PsfColCfg {
  using C = ColCfg<NY>;
  static constexpr int ACC = NY + 1;  // odd float stride: conflict-free column reads
  static constexpr size_t SMEM = ((C::SMEM + 15) & ~(size_t)15) + sizeof(float) * (size_t)C::V * ACC;
};

// Q > 0: every wavelength's pupil rows map to FFT rows within Q N/R_0 of the
// ends (checked on the host), so the first stage skips the zero inputs
template <int NY, int Q>
__global__ void __launch_bounds__(ColCfg<NY>::THREADS, ColCfg<NY>::MINB) k_psf_cols(PsfArgs a) {
  using C = ColCfg<NY>;
  constexpr int V = C::V, LEN = C::LEN, ACC = PsfColCfg<NY>::ACC;
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* tile = sm + C::TW;
  float* accs = reinterpret_cast<float*>(reinterpret_cast<char*>(sm) + ((C::SMEM + 15) & ~(size_t)15));
  load_twiddles<NY>(tw, a.twg, threadIdx.x, blockDim.x);
  const int team = threadIdx.x / C::LPV, lane = threadIdx.x % C::LPV;
  float2* s = tile + team * LEN;
  float* acc = accs + team * ACC;
  const int tiles_x = (a.nx + V - 1) / V;
  const long total = (long)tiles_x * a.zc;
  for (long t = blockIdx.x; t < total; t += gridDim.x) {
    const int zl = (int)(t / tiles_x);
    const int x0 = (int)(t % tiles_x) * V;
    for (int w = 0; w < a.W; ++w) {
      const PsfWv& p = a.wv[w];
      const float dens = (float)p.dens;
      const float2* src = a.T + ((size_t)zl * a.rowsum + a.prefix[w]) * a.nx;
      const int ylo = a.ylo[w];
      const int slo = support_lo(a, w), shi = support_hi(a, w);
      __syncthreads();
      // field rows [slo, shi) feed FFT rows (y - ny/2) mod ny (ifftshift)
      load_col_tile<V, LEN>(tile, src - (size_t)ylo * a.nx, a.nx, x0, a.nx, slo, shi,
                            [&](int y) { return add_mod(y, NY - NY / 2, NY); });
      __syncthreads();
      // FFT row n holds field row (n + NY/2) mod NY; the support [slo, shi)
      // contains the centre row NY/2 (or is empty), so it maps to
      // n < shi - NY/2 or n >= slo + NY - NY/2
      const int n_lo = shi - NY / 2, n_hi = slo + (NY - NY / 2);
      auto load = [&](int n) -> float2 {
        return (n < n_lo || n >= n_hi) ? s[pad_idx(n)] : make_float2(0.f, 0.f);
      };
      auto store = [&](int k, float2 v, int) {
        const float e = dens * cabs2(v);
        acc[k] = (w == 0) ? e : acc[k] + e;
      };
      team_fft<NY, false, C::LPV, C::CTA, (Q > 0 ? edge_zero_mask<NY, Q>() : 0u)>(s, tw, lane, team, load, store);
    }
    __syncthreads();
    float* outz = a.out + (size_t)(a.z0 + zl) * a.ny * a.nx;
    for (int idx = threadIdx.x; idx < a.ny * V; idx += blockDim.x) {
      const int row = idx / V, c = idx % V, x = x0 + c;
      if (x < a.nx) {
        const int k = add_mod(row, NY - NY / 2, NY);  // fftshift along y
        outz[(size_t)row * a.nx + add_mod(x, a.nx / 2, a.nx)] = accs[c * ACC + k];
      }
    }
  }
}

// accurate-mode source tables M and CX (see PsfArgs), after the count pass
__global__ void k_psf_tables(PsfArgs a);

// The pupil boxes of every wavelength (rows [ylo, ylo + nrows) or columns
// [xlo, xlo + ncols) of a length-n axis) map, after the ifftshift, to FFT
// indices within q n / r0 of both ends
inline bool psf_edges_within(const PsfArgs& a, bool rows, int n, int r0, int q) {
  const long lim = (long)q * (n / r0);
  for (int w = 0; w < a.W; ++w) {
    const long lo = rows ? a.ylo[w] : a.xlo[w];
    const long hi = lo + (rows ? a.nrows[w] : a.ncols[w]);  // exclusive
    if (hi - n / 2 > lim || n / 2 - lo > lim) return false;
  }
  return true;
}

// the narrowest first-stage band (in units of N / R_0 from each end) that
// holds every wavelength's pupil box: 3, 4 or 6, else 0 (dense)
inline int psf_edge_q(const PsfArgs& a, bool rows, int n, int r0) {
  if (r0 < 16) return 0;
  for (int q : {3, 4, 6})
    if (psf_edges_within(a, rows, n, r0, q)) return q;
  return 0;
}

cx_status psf_dispatch_rows(int n, const PsfArgs& a, cudaStream_t st);
cx_status psf_dispatch_cols(int n, const PsfArgs& a, cudaStream_t st);
// CX_PREC_SPLIT16 column pass on the tensor cores (psf_tc.cu)
bool psf_tc_supported(int ny, int nx);
cx_status psf_dispatch_cols_tc(int n, const PsfArgs& a, cudaStream_t st);
inline cx_status psf_cols(const PsfArgs& a, cudaStream_t st) {
  return a.precision == CX_PREC_SPLIT16 ? psf_dispatch_cols_tc(a.ny, a, st) : psf_dispatch_cols(a.ny, a, st);
}
// CX_PREC_SPLIT16 row pass on the tensor cores where the row length is
// compiled in (1024, 1280); other lengths keep the FP32 butterflies
bool psf_tc_rows_supported(int nx);
cx_status psf_dispatch_rows_tc(int n, const PsfArgs& a, cudaStream_t st);
inline cx_status psf_rows_pass(const PsfArgs& a, cudaStream_t st) {
  return a.precision == CX_PREC_SPLIT16 && psf_tc_rows_supported(a.nx) ? psf_dispatch_rows_tc(a.nx, a, st)
                                                                        : psf_dispatch_rows(a.nx, a, st);
}
}  // namespace cx
