// High-NA lens (functional/lenses.py:98-156): the defocus multiplier
// exp(i k sz f) / sz on the pupil's frequency grid and, for vector fields,
// the spherical basis change of core/field.py:897-940 in one pass over the
// pupil, then the zoomed FFT (utils/czt.py:83-124) as two chirp-Z passes
// (y, then x) with the fused Bluestein kernels of cx_czt.
#include <cmath>

#include "host.cuh"

namespace cx {

struct HighNaArgs {
  int n_fields, ny, nx, P;    // P: 1 (scalar) or 3 (vector, components z, y, x)
  double kf;                  // k f, k = 2 pi n / lambda
  double c_s;                 // NA^2 (lambda / n)^2: sz^2 = 1 - c_s (fy^2 + fx^2)
  double fy_step, fx_step;    // 1 / (ny dy), 1 / (nx dx)
  double dy, dx, oy, ox;      // spatial grid dx (i - N/2) + origin
  double r2max, inv_f2;       // (f NA / n)^2, 1 / f^2
};

// One pupil pixel per thread.  FP64 multiplier and basis change (the phase
// k sz f reaches 1e4 rad for millimetre focal lengths); the field itself is
// float32.
__global__ void k_high_na_pupil(HighNaArgs a, const float2* __restrict__ u, float2* __restrict__ out) {
  const long total = (long)a.n_fields * a.ny * a.nx;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int ix = (int)(i % a.nx), iy = (int)((i / a.nx) % a.ny);
    // frequency grid fftshift(fftfreq(N)) / dx = (i - N // 2) / (N dx)
    const double fy = (double)(iy - a.ny / 2) * a.fy_step, fx = (double)(ix - a.nx / 2) * a.fx_step;
    const double sz = sqrt(fmax(1.0 - a.c_s * (fy * fy + fx * fx), 0.0));
    double dr = 0.0, di = 0.0;
    if (sz != 0.0) {
      // FP64 phase k f sz reduced mod 2 pi in FP64, FP32 sin / cos
      const float2 e = expi_reduced(a.kf * sz);
      dr = (double)e.x / sz;
      di = (double)e.y / sz;
    }
    if (a.P == 1) {
      const float2 v = u[i];
      out[i] = make_float2((float)(v.x * dr - v.y * di), (float)(v.x * di + v.y * dr));
      continue;
    }
    const double gy = ((double)iy - 0.5 * a.ny) * a.dy + a.oy, gx = ((double)ix - 0.5 * a.nx) * a.dx + a.ox;
    const double r2 = gy * gy + gx * gx;
    const double st2 = r2 <= a.r2max ? r2 * a.inv_f2 : 0.0;
    const double ct = sqrt(1.0 - st2), st = sqrt(st2);
    double sp, cp;
    sincos(atan2(gy, gx), &sp, &cp);
    const double s2p = 2.0 * sp * cp, c2p = cp * cp - sp * sp;
    const float2 ux = u[3 * i + 2], uy = u[3 * i + 1];
    // (e_z, e_y, e_x) / 2 with real coefficients
    const double axx = 0.5 * ((ct + 1.0) + (ct - 1.0) * c2p), axy = 0.5 * (ct - 1.0) * s2p;
    const double ayy = 0.5 * ((ct + 1.0) - (ct - 1.0) * c2p);
    const double azx = -st * cp, azy = -st * sp;
    const double ex_r = axx * ux.x + axy * uy.x, ex_i = axx * ux.y + axy * uy.y;
    const double ey_r = ayy * uy.x + axy * ux.x, ey_i = ayy * uy.y + axy * ux.y;
    const double ez_r = azx * ux.x + azy * uy.x, ez_i = azx * ux.y + azy * uy.y;
    out[3 * i + 0] = make_float2((float)(ez_r * dr - ez_i * di), (float)(ez_r * di + ez_i * dr));
    out[3 * i + 1] = make_float2((float)(ey_r * dr - ey_i * di), (float)(ey_r * di + ey_i * dr));
    out[3 * i + 2] = make_float2((float)(ex_r * dr - ex_i * di), (float)(ex_r * di + ex_i * dr));
  }
}

struct HighNaPlan {
  HighNaArgs a;
  cx_czt_desc cy, cx_;
  size_t off_mid, off_czt, czt_bytes, total;
};

static cx_status high_na_plan(const cx_high_na_desc* d, HighNaPlan* p) {
  if (!d || d->n_fields < 1 || d->ny < 1 || d->nx < 2 || d->my < 2 || d->mx < 2 ||
      (d->vectorial != 0 && d->vectorial != 1) || !(d->f > 0) || !(d->n_medium > 0) || !(d->wavelength > 0) ||
      !(d->dy > 0) || !(d->dx > 0) || !(d->output_dx > 0)) {
    set_error("invalid high-NA lens descriptor (nx, my, mx >= 2; f, n, wavelength, spacings > 0)");
    return CX_ERR_INVALID;
  }
  const double pi = 3.141592653589793238462643383279502884;
  const int P = d->vectorial ? 3 : 1;
  HighNaArgs& a = p->a;
  a.n_fields = d->n_fields;
  a.ny = d->ny;
  a.nx = d->nx;
  a.P = P;
  a.kf = 2.0 * pi * d->n_medium / d->wavelength * d->f;
  const double ln = d->wavelength / d->n_medium;
  a.c_s = d->NA * d->NA * ln * ln;
  a.fy_step = 1.0 / (d->ny * d->dy);
  a.fx_step = 1.0 / (d->nx * d->dx);
  a.dy = d->dy;
  a.dx = d->dx;
  a.oy = d->origin_y;
  a.ox = d->origin_x;
  const double rp = d->f * d->NA / d->n_medium;
  a.r2max = rp * rp;
  a.inv_f2 = 1.0 / (d->f * d->f);
  // zoomed_fft(k_start = -zoom pi, k_end = zoom pi, include_end): a = exp(-i k_start),
  // w = exp(i (k_end - k_start) / (m - 1)); zoom = 2 NA fov_out / ((N - 1) lambda)
  const double zoom = 2.0 * d->NA * d->my * d->output_dx / ((d->nx - 1) * d->wavelength);
  const double ta = zoom * pi;
  const long nf = d->n_fields;
  cx_czt_desc cy{};
  cy.n = d->ny;
  cy.m = d->my;
  cy.inner = d->nx * P;
  cy.n_vec = nf * d->nx * P;
  cy.in_ostride = (int64_t)d->ny * d->nx * P;
  cy.in_istride = 1;
  cy.in_estride = (int64_t)d->nx * P;
  cy.out_ostride = (int64_t)d->my * d->nx * P;
  cy.out_istride = 1;
  cy.out_estride = (int64_t)d->nx * P;
  cy.a_re = std::cos(ta);
  cy.a_im = std::sin(ta);
  cy.w_re = std::cos(2.0 * ta / (d->my - 1));
  cy.w_im = std::sin(2.0 * ta / (d->my - 1));
  cy.mod_n = -1;
  cy.layout = 1;
  cy.scale = 1.0;
  cx_czt_desc cx2 = cy;
  cx2.n = d->nx;
  cx2.m = d->mx;
  cx2.inner = P;
  cx2.n_vec = nf * d->my * P;
  cx2.in_ostride = (int64_t)d->nx * P;
  cx2.in_estride = P;
  cx2.out_ostride = (int64_t)d->mx * P;
  cx2.out_estride = P;
  cx2.w_re = std::cos(2.0 * ta / (d->mx - 1));
  cx2.w_im = std::sin(2.0 * ta / (d->mx - 1));
  cx2.layout = P > 1 ? 1 : 0;
  p->cy = cy;
  p->cx_ = cx2;
  size_t wy = 0, wx = 0;
  cx_status s;
  if ((s = cx_czt_workspace_size(&p->cy, &wy)) != CX_OK) return s;
  if ((s = cx_czt_workspace_size(&p->cx_, &wx)) != CX_OK) return s;
  auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
  p->off_mid = al(sizeof(float2) * (size_t)nf * d->ny * d->nx * P);
  p->off_czt = p->off_mid + al(sizeof(float2) * (size_t)nf * d->my * d->nx * P);
  p->czt_bytes = wy > wx ? wy : wx;
  p->total = p->off_czt + al(p->czt_bytes);
  return CX_OK;
}

}  // namespace cx

using namespace cx;

extern "C" cx_status cx_high_na_ff_lens_workspace_size(const cx_high_na_desc* d, size_t* bytes) {
  HighNaPlan p;
  cx_status s = high_na_plan(d, &p);
  if (s != CX_OK) return s;
  if (!bytes) return CX_ERR_INVALID;
  *bytes = p.total;
  return CX_OK;
}

extern "C" cx_status cx_high_na_ff_lens(const cx_high_na_desc* d, const void* u_in, void* u_out, void* workspace,
                                        size_t workspace_bytes, cx_stream_t stream) {
  HighNaPlan p;
  cx_status s = high_na_plan(d, &p);
  if (s != CX_OK) return s;
  if (!u_in || !u_out || !workspace) {
    set_error("null pointer argument");
    return CX_ERR_INVALID;
  }
  if (workspace_bytes < p.total) {
    set_error("workspace too small: %zu < %zu", workspace_bytes, p.total);
    return CX_ERR_WORKSPACE;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  char* ws = static_cast<char*>(workspace);
  float2* pupil = reinterpret_cast<float2*>(ws);
  float2* mid = reinterpret_cast<float2*>(ws + p.off_mid);
  const long total = (long)d->n_fields * d->ny * d->nx;
  const int blocks = (int)((total + 255) / 256 < 148L * 16 ? (total + 255) / 256 : 148L * 16);
  k_high_na_pupil<<<blocks, 256, 0, st>>>(p.a, static_cast<const float2*>(u_in), pupil);
  CX_LAUNCH_CHECK();
  if ((s = cx_czt(&p.cy, pupil, mid, ws + p.off_czt, p.czt_bytes, stream)) != CX_OK) return s;
  return cx_czt(&p.cx_, mid, u_out, ws + p.off_czt, p.czt_bytes, stream);
}
