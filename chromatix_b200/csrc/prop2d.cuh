// Fourier-multiplier propagation: transfer / angular-spectrum / explicit kernel.
//
// Reference: functional/propagation.py:168-352 (transfer_propagate,
// asm_propagate), 355-394 (kernel_propagate FFT branch), 466-580
// (compute_transfer_propagator, compute_asm_propagator).
//
// Three passes over the padded (py, px) grid:
//   A  row FFT of the ny input rows, zero padding done in the loader
//      (rows outside the data are never materialised);
//   B  per V-column tile: column FFT -> x H(ky, kx) evaluated on the fly ->
//      column IFFT -> 1/(py px), only the output rows are written back;
//   C  row IFFT of the output rows, crop done in the store.
#pragma once
#include "host.cuh"

namespace cx {

struct Prop2DArgs {
  int ny, nx, py, px, pad_y, pad_x, W;
  int n_in_planes, n_out_planes;
  int out_y0, out_ny, out_x0, out_nx;
  int kernel, precision, remove_evanescent, bandlimit;
  double n_med, ky0, kx0;
  double na_f2;  // >= 0: k-space NA mask |f|^2 <= na_f2 (samples.py:276-280); < 0: none
  int precise;   // 1: FP64 sin/cos (tables reused many times); 0: FP64 reduction + hardware sin/cos
  int conj_h;    // 1: use conj(H) (adjoint passes; any kernel kind)
  const cx_plane* planes;
  const float2* H;
  const float2* twg;  // device twiddle tables (ensure_twiddles)
  // optional per-batch-element field pointers (cx_prop2d_ptrs): element b of
  // the input / output batch at in_ptrs[b] / out_ptrs[b] instead of at a
  // fixed stride from one base pointer
  const float2* const* in_ptrs = nullptr;
  float2* const* out_ptrs = nullptr;
};

// --------------------------------------------------------------------------
// the propagator H(ky, kx) in FFT bin order (already "ifftshifted")
// --------------------------------------------------------------------------
__device__ __forceinline__ float2 prop_kernel_accurate(int ky, int kx, const Prop2DArgs& a, const cx_plane& pl) {
  const double pi = 3.141592653589793238462643383279502884;
  const double K = 2.0 * pi * fabs(pl.z) * a.n_med / pl.wavelength;  // largest ASM phase (rad)
  if (!a.precise && a.kernel == CX_KERNEL_ASM && K <= 8.0 && !a.bandlimit && pl.shift_y == 0.0 &&
      pl.shift_x == 0.0) {
    // Short distances (thin slices): every phase term is below 8 rad, so FP32
    // square root and sin / cos keep the phase error below ~1e-6 rad -- inside
    // the accuracy budget -- at a fraction of the FP64 cost.  kern = 1 - q^2 f^2
    // is formed in FP64: in FP32 it cancels near the evanescent boundary
    // (kern -> 0), where sqrt(kern) magnifies the rounding into ~1e-4 rad.
    const double fy = (double)freq_index(ky, a.py) / ((double)a.py * pl.dy) - a.ky0;
    const double fx = (double)freq_index(kx, a.px) / ((double)a.px * pl.dx) - a.kx0;
    const double q = pl.wavelength / a.n_med;
    const float kern = (float)(1.0 - (q * q) * (fy * fy + fx * fx));
    float amp = 1.f, ph = 0.f;
    if (kern >= 0.f || a.remove_evanescent) {
      ph = (float)K * sqrtf(fmaxf(kern, 0.f));
    } else {
      amp = __expf(-(float)K * sqrtf(-kern));
    }
    float sn, cs;
    __sincosf(ph - 6.2831853071795865f * rintf(ph * 0.15915494309189534f), &sn, &cs);
    if (pl.z < 0.0) sn = -sn;
    return make_float2(amp * cs, amp * sn);
  }
  const double fy = (double)freq_index(ky, a.py) / ((double)a.py * pl.dy);
  const double fx = (double)freq_index(kx, a.px) / ((double)a.px * pl.dx);
  if (a.kernel == CX_KERNEL_SAS) {
    // Delta H = W exp(i kz (H_AS - H_Fr)), s = lam f / n, W the band limit
    // s^2 (2 + 1/t^2) <= 1 per axis with t = extent / |z| + |s| (propagation.py:85-103)
    const double lam = pl.wavelength, n = a.n_med;
    const double sy = lam * fy / n, sx = lam * fx / n;
    const double ty = (double)a.py * pl.dy / fabs(pl.z) + fabs(sy);
    const double tx = (double)a.px * pl.dx / fabs(pl.z) + fabs(sx);
    if (!(sy * sy * (2.0 + 1.0 / (ty * ty)) <= 1.0) || !(sx * sx * (2.0 + 1.0 / (tx * tx)) <= 1.0))
      return make_float2(0.f, 0.f);
    const double ss = sy * sy + sx * sx;
    const double h_as = sqrt(1.0 - ss > 0.0 ? 1.0 - ss : 0.0);
    const double h_fr = 1.0 - ss / 2.0;
    const double ph = 2.0 * pl.z * pi * n / lam * (h_as - h_fr);
    double sd, cd;
    sincos(ph, &sd, &cd);
    return make_float2((float)cd, (float)sd);
  }
  const double gy = fy - a.ky0, gx = fx - a.kx0;
  const double s = gy * gy + gx * gx;
  if (a.kernel == CX_KERNEL_TRANSFER) {
    // phase = -pi lam / n z |f - kykx|^2  (propagation.py:493-496)
    const double ph = -pi * pl.wavelength / a.n_med * pl.z * s;
    if (a.precise) {
      double sd, cd;
      sincos(ph, &sd, &cd);
      return make_float2((float)cd, (float)sd);
    }
    return expi_reduced(ph);
  }
  if (a.bandlimit && (fabs(fy - pl.bl_y0) > pl.bl_hy || fabs(fx - pl.bl_x0) > pl.bl_hx)) return make_float2(0.f, 0.f);
  const double q = pl.wavelength / a.n_med;
  const double kern = 1.0 - q * q * s;
  const double sh = 2.0 * pi * (fy * pl.shift_y + fx * pl.shift_x);
  double amp = 1.0, ph;
  if (kern >= 0.0 || a.remove_evanescent) {
    ph = K * sqrt(kern > 0.0 ? kern : 0.0) + sh;
  } else {
    amp = exp(-K * sqrt(-kern));
    ph = sh;
  }
  if (pl.z < 0.0) ph = -ph;  // conj(exp(i phase)) keeps the decay (propagation.py:556)
  if (a.precise) {
    double sd, cd;
    sincos(ph, &sd, &cd);
    return make_float2((float)(amp * cd), (float)(amp * sd));
  }
  float2 e = expi_reduced(ph);
  return make_float2((float)amp * e.x, (float)amp * e.y);
}

// float32 evaluation in the reference's operation order (no FMA contraction)
__device__ __forceinline__ float2 prop_kernel_ref32(int ky, int kx, const Prop2DArgs& a, const cx_plane& pl) {
  const float PI = 3.14159265358979323846f, TWO_PI = 6.28318530717958647692f;
  const float dyf = (float)pl.dy, dxf = (float)pl.dx;
  const float fy = fm(fd((float)freq_index(ky, a.py), (float)a.py), fd(1.f, dyf));
  const float fx = fm(fd((float)freq_index(kx, a.px), (float)a.px), fd(1.f, dxf));
  const float gy = fs(fy, (float)a.ky0), gx = fs(fx, (float)a.kx0);
  const float s = fa(fm(gy, gy), fm(gx, gx));
  const float lam = (float)pl.wavelength, n = (float)a.n_med, z = (float)pl.z;
  if (a.kernel == CX_KERNEL_SAS) {
    // float32 in the order of compute_sas_precompensation (propagation.py:90-102)
    const float kz = fd(fm(fm(fm(2.f, z), PI), n), lam);
    const float sy = fd(fm(lam, fy), n), sx = fd(fm(lam, fx), n);
    const float qy = fm(sy, sy), qx = fm(sx, sx);
    const float Ly = fm(2.f, fm((float)a.py, dyf)), Lx = fm(2.f, fm((float)a.px, dxf));
    const float ty = fa(fd(fd(Ly, 2.f), fabsf(z)), fabsf(sy)), tx = fa(fd(fd(Lx, 2.f), fabsf(z)), fabsf(sx));
    const bool wy = fm(qy, fa(2.f, fd(1.f, fm(ty, ty)))) <= 1.f;
    const bool wx = fm(qx, fa(2.f, fd(1.f, fm(tx, tx)))) <= 1.f;
    if (!(wy && wx)) return make_float2(0.f, 0.f);
    const float ss = fa(qy, qx);
    const float h_as = __fsqrt_rn(fmaxf(0.f, fs(1.f, ss)));
    const float h_fr = fs(1.f, fd(ss, 2.f));
    float sn, cs;
    sincosf(fm(kz, fs(h_as, h_fr)), &sn, &cs);
    return make_float2(cs, sn);
  }
  if (a.kernel == CX_KERNEL_TRANSFER) {
    const float ph = fm(fm(fd(fm(-PI, lam), n), z), s);
    float sn, cs;
    sincosf(ph, &sn, &cs);
    return make_float2(cs, sn);
  }
  if (a.bandlimit && (fabsf(fs(fy, (float)pl.bl_y0)) > (float)pl.bl_hy || fabsf(fs(fx, (float)pl.bl_x0)) > (float)pl.bl_hx))
    return make_float2(0.f, 0.f);
  const float q = fd(lam, n);
  const float kern = fs(1.f, fm(fm(q, q), s));
  const float A = fd(fm(fabsf(z), n), lam);
  const float c = fm(TWO_PI, A);
  const float sh = fm(TWO_PI, fa(fm(fy, (float)pl.shift_y), fm(fx, (float)pl.shift_x)));
  float amp = 1.f, ph;
  if (kern >= 0.f || a.remove_evanescent) {
    ph = fa(fm(c, __fsqrt_rn(kern > 0.f ? kern : 0.f)), sh);
  } else {
    amp = expf(-fm(c, __fsqrt_rn(-kern)));
    ph = sh;
  }
  float sn, cs;
  sincosf(ph, &sn, &cs);
  if (z < 0.f) sn = -sn;
  return make_float2(amp * cs, amp * sn);
}

__device__ __forceinline__ bool outside_na(int ky, int kx, const Prop2DArgs& a, const cx_plane& pl) {
  if (a.na_f2 < 0.0) return false;
  const double fy = (double)freq_index(ky, a.py) / ((double)a.py * pl.dy);
  const double fx = (double)freq_index(kx, a.px) / ((double)a.px * pl.dx);
  return fy * fy + fx * fx > a.na_f2;
}

__device__ __forceinline__ float2 prop_kernel(int ky, int kx, const Prop2DArgs& a, const cx_plane& pl) {
  if (outside_na(ky, kx, a, pl)) return make_float2(0.f, 0.f);
  float2 h;
  if (a.kernel == CX_KERNEL_EXPLICIT)
    h = a.H[((size_t)pl.h_plane * a.py + ky) * a.px + kx];
  else
    h = a.precision == CX_PREC_REF32 ? prop_kernel_ref32(ky, kx, a, pl) : prop_kernel_accurate(ky, kx, a, pl);
  return a.conj_h ? cconj(h) : h;
}

// Per-plane constants of the accurate propagator, formed once per plane (per
// column tile) instead of per element: the frequency steps as reciprocals
// (f = k * (1 / (N d)) is within an ulp of k / (N d)), the ASM phase scale
// K = 2 pi |z| n / lambda, (lambda / n)^2 and the Fresnel phase factor.
struct PropK {
  double iy, ix, K, q2, tz;
  int fast;     // the short-distance FP32 branch of prop_kernel_accurate applies
  int shifted;  // the plane has a nonzero output shift (linear phase term)
};

__device__ __forceinline__ PropK prop_consts(const Prop2DArgs& a, const cx_plane& pl) {
  const double pi = 3.141592653589793238462643383279502884;
  PropK c;
  c.iy = 1.0 / ((double)a.py * pl.dy);
  c.ix = 1.0 / ((double)a.px * pl.dx);
  c.K = 2.0 * pi * fabs(pl.z) * a.n_med / pl.wavelength;
  const double q = pl.wavelength / a.n_med;
  c.q2 = q * q;
  c.tz = -pi * pl.wavelength / a.n_med * pl.z;
  c.fast = (!a.precise && a.kernel == CX_KERNEL_ASM && c.K <= 8.0 && !a.bandlimit && pl.shift_y == 0.0 &&
            pl.shift_x == 0.0)
               ? 1
               : 0;
  c.shifted = (pl.shift_y != 0.0 || pl.shift_x != 0.0) ? 1 : 0;
  return c;
}

// sqrt(x) for 0 <= x <= 1 to FP64 accuracy from the FP32 hardware estimate
// and one Newton-Raphson (Heron) step in FP64:
//   s0 = x_f rsqrt(x_f),  s1 = s0 + (x - s0^2) / (2 s0),
// with 1 / s0 taken from the same FP32 reciprocal square root.  s0 carries
// a relative error e ~ 1e-7, so s1 is within ~e^2 + e * |x - s0^2| / s0 ~ 1e-14
// of sqrt(x) relatively (the ASM phase K sqrt(.) with K <= 1e5 rad then stays
// within 1e-9 rad).  x below the smallest normal float gives 0 (its root,
// < 1e-19, times K is far below the phase budget).
__device__ __forceinline__ double sqrt_unit_f64(double x) {
  const float xf = (float)x;
  if (!(xf > 0.f)) return 0.0;
  const float r = rsqrtf(xf);
  const double s0 = (double)(xf * r);
  return fma(fma(-s0, s0, x), 0.5 * (double)r, s0);
}

// prop_kernel_accurate for the transfer and ASM kinds with the per-plane
// constants hoisted (same branches and operation order otherwise; the FP64
// square root by sqrt_unit_f64)
__device__ __forceinline__ float2 prop_kernel_accurate_k(int ky, int kx, const Prop2DArgs& a, const cx_plane& pl,
                                                         const PropK& c) {
  const double pi = 3.141592653589793238462643383279502884;
  const double fy = (double)freq_index(ky, a.py) * c.iy;
  const double fx = (double)freq_index(kx, a.px) * c.ix;
  if (c.fast) {
    const double gy = fy - a.ky0, gx = fx - a.kx0;
    const float kern = (float)(1.0 - c.q2 * (gy * gy + gx * gx));
    float amp = 1.f, ph = 0.f;
    if (kern >= 0.f || a.remove_evanescent) {
      ph = (float)c.K * sqrtf(fmaxf(kern, 0.f));
    } else {
      amp = __expf(-(float)c.K * sqrtf(-kern));
    }
    float sn, cs;
    __sincosf(ph - 6.2831853071795865f * rintf(ph * 0.15915494309189534f), &sn, &cs);
    if (pl.z < 0.0) sn = -sn;
    return make_float2(amp * cs, amp * sn);
  }
  const double gy = fy - a.ky0, gx = fx - a.kx0;
  const double s = gy * gy + gx * gx;
  if (a.kernel == CX_KERNEL_TRANSFER) {
    const double ph = c.tz * s;
    if (a.precise) {
      double sd, cd;
      sincos(ph, &sd, &cd);
      return make_float2((float)cd, (float)sd);
    }
    return expi_reduced(ph);
  }
  if (a.bandlimit && (fabs(fy - pl.bl_y0) > pl.bl_hy || fabs(fx - pl.bl_x0) > pl.bl_hx)) return make_float2(0.f, 0.f);
  const double kern = 1.0 - c.q2 * s;
  const double sh = c.shifted ? 2.0 * pi * (fy * pl.shift_y + fx * pl.shift_x) : 0.0;
  double amp = 1.0, ph;
  if (kern >= 0.0 || a.remove_evanescent) {
    ph = c.K * sqrt_unit_f64(kern) + sh;
  } else {
    amp = exp(-c.K * sqrt_unit_f64(-kern));
    ph = sh;
  }
  if (pl.z < 0.0) ph = -ph;
  if (a.precise) {
    double sd, cd;
    sincos(ph, &sd, &cd);
    return make_float2((float)(amp * cd), (float)(amp * sd));
  }
  float2 e = expi_reduced(ph);
  return make_float2((float)amp * e.x, (float)amp * e.y);
}

// prop_kernel with the per-plane constants c = prop_consts(a, pl)
__device__ __forceinline__ float2 prop_kernel_k(int ky, int kx, const Prop2DArgs& a, const cx_plane& pl,
                                                const PropK& c) {
  if (outside_na(ky, kx, a, pl)) return make_float2(0.f, 0.f);
  float2 h;
  if (a.kernel == CX_KERNEL_EXPLICIT)
    h = a.H[((size_t)pl.h_plane * a.py + ky) * a.px + kx];
  else if (a.precision == CX_PREC_REF32)
    h = prop_kernel_ref32(ky, kx, a, pl);
  else if (a.kernel == CX_KERNEL_SAS)
    h = prop_kernel_accurate(ky, kx, a, pl);
  else
    h = prop_kernel_accurate_k(ky, kx, a, pl, c);
  return a.conj_h ? cconj(h) : h;
}

// The propagator along one column kx, specialised once per tile: the
// accurate ASM (long-distance FP64 phase, or the short-distance FP32 branch)
// and transfer kernels without NA mask or band limit take a branch-light
// path with the column's (f_x - k_x0)^2 formed once and the conjugations
// (z < 0, conj_h) folded into one sign; everything else goes through
// prop_kernel_k.  Values equal prop_kernel_k's up to the rounding of the
// re-associated sums.
struct PropCol {
  int mode;    // 0 generic, 1 ASM (FP64 phase), 2 transfer, 3 ASM short-distance branch, 4 table
  float sgn;   // sign of the phase (z < 0 and conj_h each flip it; transfer: conj_h only)
  double fx, gx2;
};

__device__ __forceinline__ PropCol prop_col(const Prop2DArgs& a, const cx_plane& pl, const PropK& c, int kx) {
  PropCol pc;
  pc.fx = (double)freq_index(kx, a.px) * c.ix;
  const double gx = pc.fx - a.kx0;
  pc.gx2 = gx * gx;
  const bool plain = a.precision == CX_PREC_ACCURATE && !a.precise && a.na_f2 < 0.0 && a.kernel != CX_KERNEL_EXPLICIT;
  pc.mode = (a.kernel == CX_KERNEL_EXPLICIT && a.na_f2 < 0.0) ? 4 : 0;
  if (plain && a.kernel == CX_KERNEL_TRANSFER) pc.mode = 2;
  if (plain && a.kernel == CX_KERNEL_ASM && !a.bandlimit) pc.mode = c.fast ? 3 : 1;
  const float cj = a.conj_h ? -1.f : 1.f;
  pc.sgn = (pc.mode == 2 || pc.mode == 4) ? cj : (pl.z < 0.0 ? -cj : cj);
  return pc;
}

__device__ __forceinline__ float2 prop_col_h(int ky, int kx, const PropCol& pc, const Prop2DArgs& a,
                                             const cx_plane& pl, const PropK& c) {
  const double pi = 3.141592653589793238462643383279502884;
  const double fy = (double)freq_index(ky, a.py) * c.iy;
  const double gy = fy - a.ky0;
  switch (pc.mode) {
    case 1: {
      const double kern = 1.0 - c.q2 * (gy * gy + pc.gx2);
      const double sh = c.shifted ? 2.0 * pi * (fy * pl.shift_y + pc.fx * pl.shift_x) : 0.0;
      double amp = 1.0, ph = sh;
      if (kern >= 0.0 || a.remove_evanescent)
        ph += c.K * sqrt_unit_f64(kern);
      else
        amp = exp(-c.K * sqrt_unit_f64(-kern));
      const float2 e = expi_reduced(ph);
      return make_float2((float)amp * e.x, (float)amp * pc.sgn * e.y);
    }
    case 2: {
      const float2 e = expi_reduced(c.tz * (gy * gy + pc.gx2));
      return make_float2(e.x, pc.sgn * e.y);
    }
    case 3: {
      const float kern = (float)(1.0 - c.q2 * (gy * gy + pc.gx2));
      float amp = 1.f, ph = 0.f;
      if (kern >= 0.f || a.remove_evanescent)
        ph = (float)c.K * sqrtf(fmaxf(kern, 0.f));
      else
        amp = __expf(-(float)c.K * sqrtf(-kern));
      float sn, cs;
      __sincosf(ph - 6.2831853071795865f * rintf(ph * 0.15915494309189534f), &sn, &cs);
      return make_float2(amp * cs, amp * pc.sgn * sn);
    }
    case 4: {
      const float2 h = a.H[((size_t)pl.h_plane * a.py + ky) * a.px + kx];
      return make_float2(h.x, pc.sgn * h.y);
    }
    default:
      return prop_kernel_k(ky, kx, a, pl, c);
  }
}

// --------------------------------------------------------------------------
// pass A: forward row FFT with zero padding in the loader
// --------------------------------------------------------------------------
// BAND: the data columns lie in [NX / 4, 3 NX / 4) (checked on the host), so
// the first stage skips the zero padding outside that band (center_band_mask)
template <int NX, bool BAND = false>
__global__ void __launch_bounds__(RowCfg<NX>::THREADS, RowCfg<NX>::MINB) k_prop_rows_fwd(const float2* __restrict__ u,
                                                                      float2* __restrict__ T, Prop2DArgs a) {
  using C = RowCfg<NX>;
  extern __shared__ float2 sm[];
  float2* tw = sm;
  load_twiddles<NX>(tw, a.twg, threadIdx.x, blockDim.x);
  __syncthreads();
  const int team = threadIdx.x / C::LPV, lane = threadIdx.x % C::LPV;
  float2* s = sm + C::TW + team * Plan<NX>::LEN;
  const long total = (long)a.n_in_planes * a.ny;
  for (long base = (long)blockIdx.x * C::TEAMS; base < total; base += (long)gridDim.x * C::TEAMS) {
    const long item = base + team;
    const bool valid = item < total;
    const int p = valid ? (int)(item / a.ny) : 0;
    const int y = valid ? (int)(item % a.ny) : 0;
    const int b = p / a.W, w = p % a.W;
    const float2* ub = a.in_ptrs ? (valid ? a.in_ptrs[b] : a.in_ptrs[0]) : u + (size_t)b * a.ny * a.nx * a.W;
    const float2* src = ub + (size_t)y * a.nx * a.W + w;
    float2* dst = T + ((size_t)p * a.ny + y) * a.px;
    auto load = [&](int n) -> float2 {
      const int x = n - a.pad_x;
      return (valid && x >= 0 && x < a.nx) ? src[(size_t)x * a.W] : make_float2(0.f, 0.f);
    };
    auto store = [&](int k, float2 v, int) {
      if (valid) dst[k] = v;
    };
    team_fft<NX, false, Plan<NX>::LPV, false, (BAND ? center_band_mask<NX>() : 0u)>(s, tw, lane, team, load, store);
  }
}

// --------------------------------------------------------------------------
// pass B: column FFT -> x H -> column IFFT on V-column tiles
// --------------------------------------------------------------------------
// BAND: the data rows lie in [NY / 4, 3 NY / 4) of the padded column (checked
// on the host), so the forward transform's first stage skips the padding.
// HT: the propagator is a table (CX_KERNEL_EXPLICIT without NA mask, e.g. the
// multislice slice propagator): the tile's V columns of H are copied into
// shared memory (cp.async) together with the data tile, instead of being read
// from global memory per element in the transform's last stage.
template <int NY>
struct PropColHt {
  static constexpr size_t SMEM = ColCfg<NY>::SMEM + sizeof(float2) * (size_t)ColCfg<NY>::V * NY;
  static constexpr bool FITS = SMEM <= 227 * 1024;
};

template <int NY, bool BAND = false, bool HT = false>
__global__ void __launch_bounds__(ColCfg<NY>::THREADS, ColCfg<NY>::MINB) k_prop_cols(const float2* __restrict__ T,
                                                                  float2* __restrict__ T2, Prop2DArgs a) {
  using C = ColCfg<NY>;
  constexpr int V = C::V, LEN = C::LEN;
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* tile = sm + C::TW;
  float2* hs = tile + V * LEN;  // HT: [V][NY] propagator columns of the tile
  load_twiddles<NY>(tw, a.twg, threadIdx.x, blockDim.x);
  const int team = threadIdx.x / C::LPV, lane = threadIdx.x % C::LPV;
  float2* s = tile + team * LEN;
  const int tiles_x = (a.px + V - 1) / V;
  const long total = (long)tiles_x * a.n_out_planes;
  const float scale = 1.0f / ((float)a.py * (float)a.px);
  for (long t = blockIdx.x; t < total; t += gridDim.x) {
    const int q = (int)(t / tiles_x);
    const int x0 = (int)(t % tiles_x) * V;
    const cx_plane pl = a.planes[q];
    const PropK kc = prop_consts(a, pl);
    const int p_in = pl.in_plane;
    __syncthreads();
    if constexpr (HT) {
      const float2* Hp = a.H + (size_t)pl.h_plane * a.py * a.px + x0;
      for (int idx = threadIdx.x; idx < NY * V; idx += blockDim.x) {
        const int r = idx / V, c = idx % V;
        if (x0 + c < a.px) cp_async8(hs + c * NY + r, Hp + (size_t)r * a.px + c);
      }
      cp_async_commit();
    }
    // cooperative, coalesced load of the ny data rows of this column tile
    load_col_tile<V, LEN>(tile, T + (size_t)p_in * a.ny * a.px, a.px, x0, a.px, 0, a.ny,
                          [&](int r) { return r + a.pad_y; });
    if constexpr (HT) cp_async_wait_all();
    __syncthreads();
    const int kx = x0 + team;
    const bool valid = kx < a.px;
    const PropCol pc = prop_col(a, pl, kc, kx);
    auto load1 = [&](int n) -> float2 {
      return (n >= a.pad_y && n < a.pad_y + a.ny) ? s[pad_idx(n)] : make_float2(0.f, 0.f);
    };
    const float2* hcol = hs + team * NY;
    auto store1 = [&](int k, float2 v, int) {
      if constexpr (HT) {
        const float2 h = hcol[k];
        s[pad_idx(k)] = valid ? cmul(v, make_float2(h.x, pc.sgn * h.y)) : v;
      } else {
        s[pad_idx(k)] = valid ? cmul(v, prop_col_h(k, kx, pc, a, pl, kc)) : v;
      }
    };
    team_fft_ex<NY, false, false, true, C::LPV, C::CTA, (BAND ? center_band_mask<NY>() : 0u)>(s, tw, lane, team,
                                                                                              load1, store1);
    team_barrier<C::LPV, C::CTA>(team);
    auto load2 = [&](int n) -> float2 { return s[pad_idx(n)]; };
    auto store2 = [&](int k, float2 v, int) { s[pad_idx(k)] = cscale(v, scale); };
    team_fft<NY, true, C::LPV, C::CTA>(s, tw, lane, team, load2, store2);
    __syncthreads();
    for (int idx = threadIdx.x; idx < a.out_ny * V; idx += blockDim.x) {
      const int r = idx / V, c = idx % V, x = x0 + c;
      if (x < a.px) T2[((size_t)q * a.out_ny + r) * a.px + x] = tile[c * LEN + pad_idx(a.out_y0 + r)];
    }
  }
}

// --------------------------------------------------------------------------
// pass C: inverse row FFT of the output rows, crop in the store
// --------------------------------------------------------------------------
template <int NX>
__global__ void __launch_bounds__(RowCfg<NX>::THREADS, RowCfg<NX>::MINB) k_prop_rows_inv(const float2* __restrict__ T2,
                                                                      float2* __restrict__ out, Prop2DArgs a) {
  using C = RowCfg<NX>;
  extern __shared__ float2 sm[];
  float2* tw = sm;
  load_twiddles<NX>(tw, a.twg, threadIdx.x, blockDim.x);
  __syncthreads();
  const int team = threadIdx.x / C::LPV, lane = threadIdx.x % C::LPV;
  float2* s = sm + C::TW + team * Plan<NX>::LEN;
  const long total = (long)a.n_out_planes * a.out_ny;
  for (long base = (long)blockIdx.x * C::TEAMS; base < total; base += (long)gridDim.x * C::TEAMS) {
    const long item = base + team;
    const bool valid = item < total;
    const int q = valid ? (int)(item / a.out_ny) : 0;
    const int r = valid ? (int)(item % a.out_ny) : 0;
    const int b = q / a.W, w = q % a.W;
    const float2* src = T2 + ((size_t)q * a.out_ny + r) * a.px;
    float2* ob = a.out_ptrs ? (valid ? a.out_ptrs[b] : a.out_ptrs[0]) : out + (size_t)b * a.out_ny * a.out_nx * a.W;
    float2* dst = ob + (size_t)r * a.out_nx * a.W + w;
    auto load = [&](int n) -> float2 { return valid ? src[n] : make_float2(0.f, 0.f); };
    auto store = [&](int k, float2 v, int) {
      const int x = k - a.out_x0;
      if (valid && x >= 0 && x < a.out_nx) dst[(size_t)x * a.W] = v;
    };
    team_fft<NX, true>(s, tw, lane, team, load, store);
  }
}

// the band variants are compiled for lengths of at least 256 whose first
// radix divides by 4; the data band [pad, pad + n) must lie in [N / 4, 3 N / 4)
template <int N>
constexpr bool band_compiled() {
  return N >= 256 && center_band_mask<N>() != 0u;
}
inline bool in_center_band(int N, int pad, int n) { return 4 * pad >= N && 4 * (pad + n) <= 3 * N; }

// dispatchers (defined in prop2d_rows.cu / prop2d_cols.cu)
cx_status dispatch_rows_fwd(int n, const float2* u, float2* T, const Prop2DArgs& a, cudaStream_t st);
cx_status dispatch_cols(int n, const float2* T, float2* T2, const Prop2DArgs& a, cudaStream_t st);
cx_status dispatch_rows_inv(int n, const float2* T2, float2* out, const Prop2DArgs& a, cudaStream_t st);
// CX_PREC_SPLIT16 column pass on the tensor cores (prop2d_tc.cu)
bool prop_tc_supported(int py, int px);
cx_status dispatch_cols_tc(int n, const float2* T, float2* T2, const Prop2DArgs& a, cudaStream_t st);
inline cx_status prop_cols(int n, const float2* T, float2* T2, const Prop2DArgs& a, cudaStream_t st) {
  return a.precision == CX_PREC_SPLIT16 ? dispatch_cols_tc(n, T, T2, a, st) : dispatch_cols(n, T, T2, a, st);
}
// CX_PREC_SPLIT16 row passes on the tensor cores where the padded row length
// is compiled in (1024, 1280); other lengths keep the FP32 butterflies
bool prop_tc_rows_supported(int px);
cx_status dispatch_rows_tc(bool inverse, const float2* in, float2* out, const Prop2DArgs& a, cudaStream_t st);
inline cx_status prop_rows_fwd(const float2* u, float2* T, const Prop2DArgs& a, cudaStream_t st) {
  return a.precision == CX_PREC_SPLIT16 && prop_tc_rows_supported(a.px) ? dispatch_rows_tc(false, u, T, a, st)
                                                                         : dispatch_rows_fwd(a.px, u, T, a, st);
}
inline cx_status prop_rows_inv(const float2* T2, float2* out, const Prop2DArgs& a, cudaStream_t st) {
  return a.precision == CX_PREC_SPLIT16 && prop_tc_rows_supported(a.px) ? dispatch_rows_tc(true, T2, out, a, st)
                                                                         : dispatch_rows_inv(a.px, T2, out, a, st);
}
}  // namespace cx
