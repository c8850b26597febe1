// Ray transfer (Collins' integral, functional/rays.py:102-154):
//   u_out = e^(i c_out |g|^2) fftshift(ifft2(ifftshift(fftshift(fft2(ifftshift(e^(i c_in |g|^2) u))) e^(-i t |f|^2))))
// with c_in = k (A - M) / (2B), c_out = k (D - 1/M) / (2B) / M^4 (the
// reference's |grid / M^2|^2), t = pi (lambda / n) B / M, k = 2 pi n / lambda.
// The centring shifts cancel around the Fourier multiplier (a convolution
// commutes with the circular shift), and e^(-i t |f|^2) is the Fresnel
// transfer function of z = B / M, so the middle is cx_prop2d's transfer
// kernel without padding; the chirps are one FP64 pass each.
#include <cmath>

#include "host.cuh"

namespace cx {

// x (n_planes interleaved as (batch, y, x, W)) times exp(i c(lambda) |g|^2),
// g = (i - N/2) d + origin, c = coef * 2 pi n / lambda
// (in may equal out: the output chirp runs in place)
__global__ void k_ray_chirp(const float2* in, float2* out, const cx_plane* __restrict__ planes,
                            int ny, int nx, int W, long total, double coef_n, double oy, double ox) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int w = (int)(i % W);
    const long pix = i / W;
    const int x = (int)(pix % nx), y = (int)((pix / nx) % ny);
    const long b = pix / ((long)nx * ny);
    const cx_plane pl = planes[b * W + w];
    const double gy = ((double)y - 0.5 * ny) * pl.dy + oy, gx = ((double)x - 0.5 * nx) * pl.dx + ox;
    // FP64 phase (it reaches 1e3..1e5 rad), reduced mod 2 pi in FP64, FP32 sin / cos
    const double ph = coef_n * 6.283185307179586476925286766559 / pl.wavelength * (gy * gy + gx * gx);
    out[i] = cmul(in[i], expi_reduced(ph));
  }
}

// the caller's planes with z = B / M (the transfer distance) and in_plane = q
__global__ void k_ray_planes(const cx_plane* __restrict__ src, cx_plane* __restrict__ dst, int n, double z) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    cx_plane p = src[q];
    p.z = z;
    p.in_plane = q;
    p.shift_y = p.shift_x = 0.0;
    dst[q] = p;
  }
}

struct RayPlan {
  cx_prop2d_desc pd;
  size_t off_planes, off_buf, off_ws, prop_ws, total;
};

static cx_status ray_plan(const cx_ray_desc* d, RayPlan* p) {
  if (!d || d->ny < 1 || d->nx < 1 || d->n_wv < 1 || d->n_planes < 1 || d->n_planes % d->n_wv ||
      !(d->n_medium > 0) || !(d->magnification != 0) || !std::isfinite(d->B)) {
    set_error("invalid ray-transfer descriptor");
    return CX_ERR_INVALID;
  }
  if (d->B == 0.0) {
    set_error("ray transfer needs B != 0 (Collins' integral divides by B)");
    return CX_ERR_INVALID;
  }
  cx_prop2d_desc& q = p->pd;
  q = cx_prop2d_desc{};
  q.ny = d->ny;
  q.nx = d->nx;
  q.n_wv = d->n_wv;
  q.n_in_planes = d->n_planes;
  q.n_out_planes = d->n_planes;
  q.mode_same = 1;
  q.kernel = CX_KERNEL_TRANSFER;
  q.precision = d->precision;
  q.n_medium = d->n_medium;
  cx_status s = cx_prop2d_workspace_size(&q, &p->prop_ws);
  if (s != CX_OK) return s;
  auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
  p->off_planes = 0;
  p->off_buf = al(sizeof(cx_plane) * (size_t)d->n_planes);
  p->off_ws = p->off_buf + al(sizeof(float2) * (size_t)d->n_planes * d->ny * d->nx);
  p->total = p->off_ws + al(p->prop_ws);
  return CX_OK;
}

}  // namespace cx

using namespace cx;

extern "C" cx_status cx_ray_transfer_workspace_size(const cx_ray_desc* d, size_t* bytes) {
  RayPlan p;
  cx_status s = ray_plan(d, &p);
  if (s != CX_OK) return s;
  if (!bytes) return CX_ERR_INVALID;
  *bytes = p.total;
  return CX_OK;
}

extern "C" cx_status cx_ray_transfer(const cx_ray_desc* d, const cx_plane* planes_dev, const void* u_in, void* u_out,
                                     void* workspace, size_t workspace_bytes, cx_stream_t stream) {
  RayPlan p;
  cx_status s = ray_plan(d, &p);
  if (s != CX_OK) return s;
  if (!planes_dev || !u_in || !u_out || !workspace) {
    set_error("null pointer argument");
    return CX_ERR_INVALID;
  }
  if (workspace_bytes < p.total) {
    set_error("workspace too small: %zu < %zu", workspace_bytes, p.total);
    return CX_ERR_WORKSPACE;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  char* ws = static_cast<char*>(workspace);
  cx_plane* pl = reinterpret_cast<cx_plane*>(ws + p.off_planes);
  float2* buf = reinterpret_cast<float2*>(ws + p.off_buf);
  const double M = d->magnification;
  k_ray_planes<<<(d->n_planes + 127) / 128, 128, 0, st>>>(planes_dev, pl, d->n_planes, d->B / M);
  CX_LAUNCH_CHECK();
  const long total = (long)(d->n_planes / d->n_wv) * d->ny * d->nx * d->n_wv;
  long g = (total + 255) / 256;
  if (g > (long)sm_count() * 16) g = (long)sm_count() * 16;
  const int grid = (int)(g < 1 ? 1 : g);
  // c = k (A - M) / (2B) with k = 2 pi n / lambda: coef_n = n (A - M) / (2B)
  const double cin = d->n_medium * (d->A - M) / (2.0 * d->B);
  const double cout = d->n_medium * (d->D - 1.0 / M) / (2.0 * d->B) / (M * M * M * M);
  k_ray_chirp<<<grid, 256, 0, st>>>(static_cast<const float2*>(u_in), buf, pl, d->ny, d->nx, d->n_wv, total, cin,
                                    d->origin_y, d->origin_x);
  CX_LAUNCH_CHECK();
  if ((s = cx_prop2d(&p.pd, pl, buf, u_out, nullptr, ws + p.off_ws, p.prop_ws, stream)) != CX_OK) return s;
  k_ray_chirp<<<grid, 256, 0, st>>>(static_cast<const float2*>(u_out), static_cast<float2*>(u_out), pl, d->ny, d->nx,
                                    d->n_wv, total, cout, d->origin_y, d->origin_x);
  CX_LAUNCH_CHECK();
  return CX_OK;
}
