// Elementwise field operations and their adjoints.
//
// Reference: functional/phase_masks.py:29-68 (phase_change),
// functional/samples.py:85-134 (thin_sample), core/field.py:656-665, 735-740
// (Field.intensity, whose adjoint is here), core/field.py:534-549 (pad with
// cval), functional/sources.py:212-293 (plane_wave), functional/pupils.py:17-67
// (circular / square / super-Gaussian / Tukey pupils).
//
// All of them are HBM-bound single passes: one read and one write of the
// field (8 B per complex value) plus the real map (4 B per pixel).  Fields
// are (n_batch, ny, nx, n_wv) complex64, the real maps (ny, nx) broadcast
// over batch and wavelength, or (n_batch, ny, nx) when map_batched.
// Threads walk the field in its memory order (coalesced); the adjoint of a
// broadcast map sums over batch and wavelength with one thread per pixel.
#include <cmath>

#include "host.cuh"

namespace cx {

static int ew_grid(long n) {
  long g = (n + 255) / 256;
  const long cap = (long)sm_count() * 8;
  if (g > cap) g = cap;
  return (int)(g < 1 ? 1 : g);
}

static cx_status ew_check(const cx_ew_desc* d) {
  if (!d || d->n_batch < 0 || d->ny <= 0 || d->nx <= 0 || d->n_wv <= 0 || d->n_wv > 64) {
    set_error("invalid elementwise descriptor (1 <= n_wv <= 64)");
    return CX_ERR_INVALID;
  }
  return CX_OK;
}

// index of the real map value of field element i = ((b ny + y) nx + x) W + w
__device__ __forceinline__ long map_index(long i, int W, long plane, int batched) {
  const long pix = i / W;  // (b ny + y) nx + x
  return batched ? pix : pix % plane;
}

// ---------------------------------------------------------------------------
// phase_change: out = u exp(i phase s_w)
// ---------------------------------------------------------------------------
__global__ void k_phase_change(const float2* __restrict__ u, const float* __restrict__ phase,
                               const float* __restrict__ s, float2* __restrict__ out, long n, int W, long plane,
                               int batched) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const int w = (int)(i % W);
    float sn, cs;
    sincosf(phase[map_index(i, W, plane, batched)] * s[w], &sn, &cs);
    out[i] = cmul(u[i], make_float2(cs, sn));
  }
}

// g_u = g exp(-i phase s_w)
__global__ void k_phase_change_gu(const float2* __restrict__ g, const float* __restrict__ phase,
                                  const float* __restrict__ s, float2* __restrict__ gu, long n, int W, long plane,
                                  int batched) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const int w = (int)(i % W);
    float sn, cs;
    sincosf(phase[map_index(i, W, plane, batched)] * s[w], &sn, &cs);
    gu[i] = cmul(g[i], make_float2(cs, -sn));
  }
}

// gradient of a real map m entering as exp(i c_w m) (c = s) or
// exp(i c_w (dn + i abs)) (thin sample):
//   d/dm  = sum_{b,w} c_w Im(g conj(out))        (phase, dn)
//   d/dabs = -sum_{b,w} c_w Re(g conj(out))      (absorption)
// one thread per map pixel; with a broadcast map it loops over the batch
__global__ void k_map_grad(const float2* __restrict__ g, const float2* __restrict__ out,
                           const float* __restrict__ c, float* __restrict__ g_im, float* __restrict__ g_re,
                           long n_map, long n_batch, int W, long plane, int batched) {
  for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < n_map; p += (long)gridDim.x * blockDim.x) {
    float acc_im = 0.f, acc_re = 0.f;
    const long nb = batched ? 1 : n_batch;
    for (long b = 0; b < nb; ++b) {
      const long base = (batched ? p : b * plane + p) * W;
      for (int w = 0; w < W; ++w) {
        const float2 gv = g[base + w], ov = out[base + w];
        // g conj(out) = (g.x o.x + g.y o.y) + i (g.y o.x - g.x o.y)
        acc_im += c[w] * (gv.y * ov.x - gv.x * ov.y);
        acc_re += c[w] * (gv.x * ov.x + gv.y * ov.y);
      }
    }
    if (g_im) g_im[p] = acc_im;
    if (g_re) g_re[p] = -acc_re;
  }
}

// ---------------------------------------------------------------------------
// thin_sample: out = u exp(i kd_w (dn + i abs)) = u exp(-kd_w abs) exp(i kd_w dn)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 transmittance(float kd, float dn, float ab, bool conj) {
  float sn, cs;
  sincosf(kd * dn, &sn, &cs);
  const float a = expf(-kd * ab);
  return make_float2(a * cs, conj ? -a * sn : a * sn);
}

__global__ void k_thin_sample(const float2* __restrict__ u, const float* __restrict__ ab,
                              const float* __restrict__ dn, const float* __restrict__ kd, float2* __restrict__ out,
                              long n, int W, long plane, int batched, int adjoint) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const int w = (int)(i % W);
    const long m = map_index(i, W, plane, batched);
    out[i] = cmul(u[i], transmittance(kd[w], dn[m], ab[m], adjoint != 0));
  }
}

// ---------------------------------------------------------------------------
// Field.intensity adjoint: g_u = 2 density_w g_I u
// ---------------------------------------------------------------------------
__global__ void k_intensity_adjoint(const float2* __restrict__ u, const float* __restrict__ gI,
                                    const double* __restrict__ density, float2* __restrict__ gu, long n, int W) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const float f = 2.f * (float)density[i % W] * gI[i / W];
    gu[i] = cscale(u[i], f);
  }
}

// ---------------------------------------------------------------------------
// pad with a constant: out (n_batch, ny + 2 py, nx + 2 px, W)
// ---------------------------------------------------------------------------
__global__ void k_pad(const float2* __restrict__ u, float2* __restrict__ out, long n_out, int ny, int nx, int oy,
                      int ox, int py, int px, int W, float2 cval) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n_out; i += (long)gridDim.x * blockDim.x) {
    const int w = (int)(i % W);
    long r = i / W;
    const int x = (int)(r % ox) - px;
    r /= ox;
    const int y = (int)(r % oy) - py;
    const long b = r / oy;
    out[i] = (y >= 0 && y < ny && x >= 0 && x < nx) ? u[((b * ny + y) * nx + x) * W + w] : cval;
  }
}

// ---------------------------------------------------------------------------
// plane_wave: u[y, x, w] = amp_w exp(i (ky gy + kx gx)), g = d_w (i - N/2)
// (+ origin); pupils: real masks on the same grid
// ---------------------------------------------------------------------------
__global__ void k_plane_wave(float2* __restrict__ u, long n, int ny, int nx, int W,
                             const double* __restrict__ wv /* (W, 3): dy, dx, amplitude */, double ky, double kx,
                             double oy, double ox) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const int w = (int)(i % W);
    const long r = i / W;
    const int x = (int)(r % nx), y = (int)((r / nx) % ny);
    const double gy = wv[3 * w] * ((double)y - 0.5 * ny) + oy;
    const double gx = wv[3 * w + 1] * ((double)x - 0.5 * nx) + ox;
    const float2 e = expi_reduced(ky * gy + kx * gx);
    const float a = (float)wv[3 * w + 2];
    u[i] = make_float2(a * e.x, a * e.y);
  }
}

// kind 0 circular |r|^2 <= p0^2; 1 square max(|y|, |x|) <= p0; 2 super-Gaussian
// exp(-(|r| / p0)^p1); 3 Tukey with alpha = p1 on r = |g / extent| (extent p2, p3)
__global__ void k_pupil(const float2* __restrict__ u, float2* __restrict__ out, long n, int ny, int nx, int W,
                        int kind, const double* __restrict__ wv /* (W, 6): dy, dx, p0, p1, p2, p3 */, double oy,
                        double ox) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const int w = (int)(i % W);
    const long r = i / W;
    const int x = (int)(r % nx), y = (int)((r / nx) % ny);
    const double* q = wv + 6 * w;
    const double gy = q[0] * ((double)y - 0.5 * ny) + oy;
    const double gx = q[1] * ((double)x - 0.5 * nx) + ox;
    double m;
    if (kind == 0) {
      m = (gy * gy + gx * gx <= q[2] * q[2]) ? 1.0 : 0.0;
    } else if (kind == 1) {
      m = (fmax(fabs(gy), fabs(gx)) <= q[2]) ? 1.0 : 0.0;
    } else if (kind == 2) {
      m = exp(-pow(sqrt(gy * gy + gx * gx) / q[2], q[3]));
    } else {
      const double ry = gy / q[4], rx = gx / q[5];
      double rr = sqrt(ry * ry + rx * rx);
      rr = rr < 0.0 ? 0.0 : (rr > 0.5 ? 0.5 : rr);
      const double alpha = q[3];
      m = rr <= alpha / 2 ? 1.0
                          : 0.5 * (1.0 + cos((2.0 * 3.141592653589793238462643383279502884 / (1.0 - alpha)) *
                                             (rr - alpha / 2)));
    }
    out[i] = cscale(u[i], (float)m);
  }
}

}  // namespace cx

using namespace cx;

extern "C" cx_status cx_phase_change(const cx_ew_desc* d, const void* u, const float* phase, const float* s_dev,
                                     void* out, cx_stream_t stream) {
  cx_status st = ew_check(d);
  if (st != CX_OK) return st;
  if (!u || !phase || !s_dev || !out) {
    set_error("cx_phase_change: null pointer argument");
    return CX_ERR_INVALID;
  }
  const long plane = (long)d->ny * d->nx, n = d->n_batch * plane * d->n_wv;
  if (n == 0) return CX_OK;
  k_phase_change<<<ew_grid(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const float2*>(u), phase, s_dev, static_cast<float2*>(out), n, d->n_wv, plane, d->map_batched);
  CX_LAUNCH_CHECK();
  return CX_OK;
}

extern "C" cx_status cx_phase_change_adjoint(const cx_ew_desc* d, const void* g, const void* out, const float* phase,
                                             const float* s_dev, void* g_u, float* g_phase, cx_stream_t stream) {
  cx_status st = ew_check(d);
  if (st != CX_OK) return st;
  if (!g || !phase || !s_dev || (g_phase && !out)) {
    set_error("cx_phase_change_adjoint: null pointer argument");
    return CX_ERR_INVALID;
  }
  const long plane = (long)d->ny * d->nx, n = d->n_batch * plane * d->n_wv;
  if (n == 0) return CX_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (g_u) {
    k_phase_change_gu<<<ew_grid(n), 256, 0, s>>>(static_cast<const float2*>(g), phase, s_dev,
                                                 static_cast<float2*>(g_u), n, d->n_wv, plane, d->map_batched);
    CX_LAUNCH_CHECK();
  }
  if (g_phase) {
    const long n_map = d->map_batched ? d->n_batch * plane : plane;
    k_map_grad<<<ew_grid(n_map), 256, 0, s>>>(static_cast<const float2*>(g), static_cast<const float2*>(out), s_dev,
                                              g_phase, nullptr, n_map, d->n_batch, d->n_wv, plane, d->map_batched);
    CX_LAUNCH_CHECK();
  }
  return CX_OK;
}

extern "C" cx_status cx_thin_sample(const cx_ew_desc* d, const void* u, const float* absorption, const float* dn,
                                    const float* kd_dev, void* out, cx_stream_t stream) {
  cx_status st = ew_check(d);
  if (st != CX_OK) return st;
  if (!u || !absorption || !dn || !kd_dev || !out) {
    set_error("cx_thin_sample: null pointer argument");
    return CX_ERR_INVALID;
  }
  const long plane = (long)d->ny * d->nx, n = d->n_batch * plane * d->n_wv;
  if (n == 0) return CX_OK;
  k_thin_sample<<<ew_grid(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const float2*>(u), absorption, dn, kd_dev, static_cast<float2*>(out), n, d->n_wv, plane,
      d->map_batched, 0);
  CX_LAUNCH_CHECK();
  return CX_OK;
}

extern "C" cx_status cx_thin_sample_adjoint(const cx_ew_desc* d, const void* g, const void* out,
                                            const float* absorption, const float* dn, const float* kd_dev, void* g_u,
                                            float* g_absorption, float* g_dn, cx_stream_t stream) {
  cx_status st = ew_check(d);
  if (st != CX_OK) return st;
  if (!g || !absorption || !dn || !kd_dev || ((g_absorption || g_dn) && !out)) {
    set_error("cx_thin_sample_adjoint: null pointer argument");
    return CX_ERR_INVALID;
  }
  const long plane = (long)d->ny * d->nx, n = d->n_batch * plane * d->n_wv;
  if (n == 0) return CX_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (g_u) {
    k_thin_sample<<<ew_grid(n), 256, 0, s>>>(static_cast<const float2*>(g), absorption, dn, kd_dev,
                                             static_cast<float2*>(g_u), n, d->n_wv, plane, d->map_batched, 1);
    CX_LAUNCH_CHECK();
  }
  if (g_absorption || g_dn) {
    const long n_map = d->map_batched ? d->n_batch * plane : plane;
    k_map_grad<<<ew_grid(n_map), 256, 0, s>>>(static_cast<const float2*>(g), static_cast<const float2*>(out), kd_dev,
                                              g_dn, g_absorption, n_map, d->n_batch, d->n_wv, plane, d->map_batched);
    CX_LAUNCH_CHECK();
  }
  return CX_OK;
}

extern "C" cx_status cx_intensity_adjoint(const void* u, int64_t n_pix, int32_t n_wv, const double* density_dev,
                                          const float* g_intensity, void* g_u, cx_stream_t stream) {
  if (!u || !g_intensity || !density_dev || !g_u || n_pix < 0 || n_wv < 1) {
    set_error("cx_intensity_adjoint: invalid arguments");
    return CX_ERR_INVALID;
  }
  const long n = (long)n_pix * n_wv;
  if (n == 0) return CX_OK;
  k_intensity_adjoint<<<ew_grid(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const float2*>(u), g_intensity, density_dev, static_cast<float2*>(g_u), n, n_wv);
  CX_LAUNCH_CHECK();
  return CX_OK;
}

extern "C" cx_status cx_pad(const cx_ew_desc* d, int32_t pad_y, int32_t pad_x, float cval_re, float cval_im,
                            const void* u, void* out, cx_stream_t stream) {
  cx_status st = ew_check(d);
  if (st != CX_OK) return st;
  if (!u || !out || pad_y < 0 || pad_x < 0) {
    set_error("cx_pad: invalid arguments");
    return CX_ERR_INVALID;
  }
  const int oy = d->ny + 2 * pad_y, ox = d->nx + 2 * pad_x;
  const long n = d->n_batch * (long)oy * ox * d->n_wv;
  if (n == 0) return CX_OK;
  k_pad<<<ew_grid(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(static_cast<const float2*>(u),
                                                                  static_cast<float2*>(out), n, d->ny, d->nx, oy, ox,
                                                                  pad_y, pad_x, d->n_wv,
                                                                  make_float2(cval_re, cval_im));
  CX_LAUNCH_CHECK();
  return CX_OK;
}

extern "C" cx_status cx_plane_wave(const cx_ew_desc* d, const double* wv_params_dev, double ky, double kx,
                                   double origin_y, double origin_x, void* u, cx_stream_t stream) {
  cx_status st = ew_check(d);
  if (st != CX_OK) return st;
  if (!u || !wv_params_dev) {
    set_error("cx_plane_wave: null pointer argument");
    return CX_ERR_INVALID;
  }
  const long n = d->n_batch * (long)d->ny * d->nx * d->n_wv;
  if (n == 0) return CX_OK;
  k_plane_wave<<<ew_grid(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(static_cast<float2*>(u), n, d->ny, d->nx,
                                                                         d->n_wv, wv_params_dev, ky, kx, origin_y,
                                                                         origin_x);
  CX_LAUNCH_CHECK();
  return CX_OK;
}

extern "C" cx_status cx_pupil(const cx_ew_desc* d, int32_t kind, const double* wv_params_dev, double origin_y,
                              double origin_x, const void* u, void* out, cx_stream_t stream) {
  cx_status st = ew_check(d);
  if (st != CX_OK) return st;
  if (!u || !out || !wv_params_dev || kind < 0 || kind > 3) {
    set_error("cx_pupil: invalid arguments");
    return CX_ERR_INVALID;
  }
  const long n = d->n_batch * (long)d->ny * d->nx * d->n_wv;
  if (n == 0) return CX_OK;
  k_pupil<<<ew_grid(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(static_cast<const float2*>(u),
                                                                    static_cast<float2*>(out), n, d->ny, d->nx,
                                                                    d->n_wv, kind, wv_params_dev, origin_y, origin_x);
  CX_LAUNCH_CHECK();
  return CX_OK;
}

// ---------------------------------------------------------------------------
// complex vector algebra for Krylov solvers (FP64 accumulation)
// ---------------------------------------------------------------------------
namespace cx {

__device__ __forceinline__ void block_add_doubles(double* v, int k, double* out) {
  __shared__ double red[4][32];
  for (int j = 0; j < k; ++j)
    for (int o = 16; o > 0; o >>= 1) v[j] += __shfl_xor_sync(0xffffffffu, v[j], o);
  const int wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  if ((threadIdx.x & 31) == 0)
    for (int j = 0; j < k; ++j) red[j][wid] = v[j];
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int j = 0; j < k; ++j) {
      double t = 0.0;
      for (int w = 0; w < nw; ++w) t += red[j][w];
      atomicAdd(out + j, t);
    }
  }
}

// out[0..1] += sum conj(x) y, out[2] += sum |x|^2, out[3] += sum |y|^2
__global__ void k_cvec_dot(const float2* __restrict__ x, const float2* __restrict__ y, long n, double* out) {
  double v[4] = {0.0, 0.0, 0.0, 0.0};
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const float2 a = x[i], b = y[i];
    v[0] += (double)a.x * b.x + (double)a.y * b.y;
    v[1] += (double)a.x * b.y - (double)a.y * b.x;
    v[2] += (double)a.x * a.x + (double)a.y * a.y;
    v[3] += (double)b.x * b.x + (double)b.y * b.y;
  }
  block_add_doubles(v, 4, out);
}

// out = ca x + cb y [+ cc z]; norm (if set) += sum |out|^2
__global__ void k_cvec_lincomb(const float2* __restrict__ x, const float2* __restrict__ y, const float2* __restrict__ z,
                               float2 ca, float2 cb, float2 cc, float2* __restrict__ out, long n, double* norm) {
  double v[1] = {0.0};
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    float2 r = cadd(cmul(ca, x[i]), cmul(cb, y[i]));
    if (z) r = cadd(r, cmul(cc, z[i]));
    out[i] = r;
    v[0] += (double)r.x * r.x + (double)r.y * r.y;
  }
  if (norm) block_add_doubles(v, 1, norm);
}

}  // namespace cx

extern "C" cx_status cx_cvec_dot(const void* x, const void* y, int64_t n, double* out_dev, cx_stream_t stream) {
  if (!x || !y || !out_dev || n < 0) {
    set_error("cx_cvec_dot: invalid arguments");
    return CX_ERR_INVALID;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  CX_CUDA_TRY(cudaMemsetAsync(out_dev, 0, 4 * sizeof(double), st));
  if (n == 0) return CX_OK;
  k_cvec_dot<<<ew_grid(n), 256, 0, st>>>(static_cast<const float2*>(x), static_cast<const float2*>(y), n, out_dev);
  CX_LAUNCH_CHECK();
  return CX_OK;
}

extern "C" cx_status cx_cvec_lincomb(int64_t n, const double* coef, const void* x, const void* y, const void* z,
                                     void* out, double* norm_dev, cx_stream_t stream) {
  if (!coef || !x || !y || !out || n < 0) {
    set_error("cx_cvec_lincomb: invalid arguments");
    return CX_ERR_INVALID;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (norm_dev) CX_CUDA_TRY(cudaMemsetAsync(norm_dev, 0, sizeof(double), st));
  if (n == 0) return CX_OK;
  k_cvec_lincomb<<<ew_grid(n), 256, 0, st>>>(
      static_cast<const float2*>(x), static_cast<const float2*>(y), static_cast<const float2*>(z),
      make_float2((float)coef[0], (float)coef[1]), make_float2((float)coef[2], (float)coef[3]),
      make_float2((float)coef[4], (float)coef[5]), static_cast<float2*>(out), n, norm_dev);
  CX_LAUNCH_CHECK();
  return CX_OK;
}

// ---------------------------------------------------------------------------
// field x planar propagator: out[b, y, x, w] = u[b, y, x, w] H[b W + w, y, x]
// (conj(H) when conj_h): the Fourier multiplier of kernel_propagate
// (functional/propagation.py:391-394) for transform lengths the fused passes
// do not cover (the transforms are then chirp-Z passes)
// ---------------------------------------------------------------------------
namespace cx {
__global__ void k_cmul_planar(const float2* __restrict__ u, const float2* __restrict__ H, float2* __restrict__ out,
                              long n, int W, long plane, int conj_h) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const int w = (int)(i % W);
    const long pix = i / W;  // b * plane + yx
    const long b = pix / plane, yx = pix - b * plane;
    float2 h = H[(b * W + w) * plane + yx];
    if (conj_h) h = cconj(h);
    out[i] = cmul(u[i], h);
  }
}
}  // namespace cx

extern "C" cx_status cx_cmul_planar(const cx_ew_desc* d, const void* u, const void* H, int32_t conj_h, void* out,
                                    cx_stream_t stream) {
  cx_status st = ew_check(d);
  if (st != CX_OK) return st;
  if (!u || !H || !out) {
    set_error("cx_cmul_planar: null pointer argument");
    return CX_ERR_INVALID;
  }
  const long plane = (long)d->ny * d->nx, n = d->n_batch * plane * d->n_wv;
  if (n == 0) return CX_OK;
  k_cmul_planar<<<ew_grid(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const float2*>(u), static_cast<const float2*>(H), static_cast<float2*>(out), n, d->n_wv, plane,
      conj_h);
  CX_LAUNCH_CHECK();
  return CX_OK;
}
