// Rescaled-output propagation (the CZT branch of kernel_propagate) in one call.
//
// Reference: functional/propagation.py:395-443 (kernel_propagate, use_czt),
// reached from transfer_propagate / asm_propagate with output_dx /
// output_shape (propagation.py:168-352).  Per field:
//   H  = propagator of the padded grid (compute_*_propagator, FFT order)
//   Y  = fftshift(H * fft2(ifftshift(pad(u))))             cx_optical_fft_h
//   Y1 = CZT_y(Y)  * w_y^(-N k) a_y^N                        column-tile CZT
//   u' = CZT_x(Y1) * w_x^(-N k) a_x^N / (alpha_y alpha_x)    row CZT
// with a = exp(-2 pi i lo / T), w = exp(2 pi i (hi - lo) / (T (m - 1))) from
// the output grid limits lo = dx_out (0 - m/2) + shift, hi = dx_out (m - 1 -
// m/2) + shift, T = dx_in * padded length and alpha = dx_out * T.  The plane
// tables the passes read are written into the workspace by a one-thread
// kernel that receives them by value, so the call needs no host-to-device
// copy and never waits on the stream.
#include <cmath>
#include <complex>

#include "czt.cuh"

namespace cx {

// finite chirp filter of the Yu et al. convolution along an axis of length n,
// arranged for the chirp-Z pass: c[i] = exp(-i pi cf (i - ic)^2) / L on
// i in [i0, i1), 0 elsewhere (FP64 phases; evaluated once per call)
__global__ void k_yu_filter(float2* __restrict__ c, int L, double cf, double ic, int i0, int i1) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < L; i += gridDim.x * blockDim.x) {
    float2 v = make_float2(0.f, 0.f);
    if (i >= i0 && i < i1) {
      const double d = (double)i - ic;
      double sd, cd;
      sincos(-3.141592653589793238462643383279502884 * cf * d * d, &sd, &cd);
      v = make_float2((float)(cd / L), (float)(sd / L));
    }
    c[i] = v;
  }
}

__global__ void k_czt_prop_tables(cx_plane* hp, cx_plane h, cx_fft_plane* fp, cx_fft_plane f) {
  if (threadIdx.x == 0) {
    *hp = h;
    *fp = f;
  }
}

struct CztPropLayout {
  int py, px, Ly, Lx;
  size_t off_h, off_y, off_t, off_c, total;
};

static size_t al256(size_t b) { return (b + 255) & ~(size_t)255; }

static int czt_len(int n, int m) {
  const int need = n + m - 1;
  for (int i = 0; i < kNumSizes; ++i)
    if (kSizes[i] >= need) return kSizes[i];
  return -1;
}

static cx_status czt_prop_layout(const cx_czt_prop_desc* d, CztPropLayout* L) {
  if (!d || d->ny <= 0 || d->nx <= 0 || d->pad_y < 0 || d->pad_x < 0 || d->my < 2 || d->mx < 2 ||
      d->n_fields <= 0 || !(d->wavelength > 0.0) || !(d->dy_in > 0.0) || !(d->dx_in > 0.0) ||
      !(d->dy_out > 0.0) || !(d->dx_out > 0.0) ||
      (d->kernel != CX_KERNEL_TRANSFER && d->kernel != CX_KERNEL_ASM)) {
    set_error("invalid rescaled-propagation descriptor (output sides >= 2, transfer or ASM kernel)");
    return CX_ERR_INVALID;
  }
  if (d->bandlimit && d->kernel != CX_KERNEL_ASM) {
    set_error("cx_czt_propagate: the band limit applies to the ASM kernel only");
    return CX_ERR_INVALID;
  }
  if (d->method != 0 && d->method != 1) {
    set_error("cx_czt_propagate: method must be 0 (chirp-Z) or 1 (Yu et al. convolution)");
    return CX_ERR_INVALID;
  }
  L->py = d->ny + 2 * d->pad_y;
  L->px = d->nx + 2 * d->pad_x;
  if (d->method == 1 && (d->my != L->py || d->mx != L->px)) {
    // the convolution keeps the padded grid (its output chirp and the "same"
    // convolution share one shape, propagation.py:452-458)
    set_error("the Yu et al. rescaling needs output_shape == padded shape (%dx%d), got %dx%d", L->py, L->px,
              d->my, d->mx);
    return CX_ERR_INVALID;
  }
  if (!size_supported(L->py) || !size_supported(L->px)) {
    set_error("padded grid %dx%d: FFT length not supported", L->py, L->px);
    return CX_ERR_UNSUPPORTED;
  }
  L->Ly = czt_len(L->py, d->my);
  L->Lx = czt_len(L->px, d->mx);
  if (L->Ly < 0 || L->Lx < 0) {
    set_error("output %dx%d from a %dx%d grid needs a CZT length above 8192", d->my, d->mx, L->py, L->px);
    return CX_ERR_UNSUPPORTED;
  }
  const size_t plane = sizeof(float2) * (size_t)L->py * L->px;
  const size_t t = sizeof(float2) * (size_t)(L->py > d->my ? L->py : d->my) * L->px;
  const int Lm = L->Ly > L->Lx ? L->Ly : L->Lx;
  L->off_h = 512;
  L->off_y = L->off_h + al256(plane);
  L->off_t = L->off_y + al256(plane);
  L->off_c = L->off_t + al256(t);
  // chirp-Z: one filter + spectrum (cx_czt's workspace); Yu: filter + spectrum per axis
  L->total = L->off_c + al256((d->method == 1 ? 4 : 2) * sizeof(float2) * (size_t)Lm);
  return CX_OK;
}

}  // namespace cx

using namespace cx;

extern "C" cx_status cx_czt_propagate_workspace_size(const cx_czt_prop_desc* d, size_t* bytes) {
  CztPropLayout L;
  cx_status s = czt_prop_layout(d, &L);
  if (s != CX_OK) return s;
  if (!bytes) return CX_ERR_INVALID;
  *bytes = L.total;
  return CX_OK;
}

extern "C" cx_status cx_czt_propagate(const cx_czt_prop_desc* d, const void* u_in, void* u_out, void* workspace,
                                      size_t workspace_bytes, cx_stream_t stream) {
  CztPropLayout L;
  cx_status s = czt_prop_layout(d, &L);
  if (s != CX_OK) return s;
  if (!u_in || !u_out || !workspace) {
    set_error("null pointer argument");
    return CX_ERR_INVALID;
  }
  if (workspace_bytes < L.total) {
    set_error("workspace too small: %zu < %zu", workspace_bytes, L.total);
    return CX_ERR_WORKSPACE;
  }
  char* ws = static_cast<char*>(workspace);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cx_plane* hp = reinterpret_cast<cx_plane*>(ws);
  cx_fft_plane* fp = reinterpret_cast<cx_fft_plane*>(ws + 256);
  float2* H = reinterpret_cast<float2*>(ws + L.off_h);
  float2* Y = reinterpret_cast<float2*>(ws + L.off_y);
  float2* T = reinterpret_cast<float2*>(ws + L.off_t);
  void* cws = ws + L.off_c;
  const size_t cws_bytes = L.total - L.off_c;

  // propagator of the padded grid with the field's spacing; with chirp-Z
  // transforms the output shift lives in their grid, not in H (propagation.py:420-443)
  cx_plane h{};
  h.z = d->z;
  h.wavelength = d->wavelength;
  h.dy = d->dy_in;
  h.dx = d->dx_in;
  if (d->bandlimit) {
    h.bl_y0 = d->bl_y0;
    h.bl_x0 = d->bl_x0;
    h.bl_hy = d->bl_hy;
    h.bl_hx = d->bl_hx;
  }
  if (d->method == 1 && d->kernel == CX_KERNEL_ASM) {
    // without the chirp-Z grid the ASM shift term stays in the propagator
    // (asm_propagate passes shift_yx unless use_czt, propagation.py:331-339)
    h.shift_y = d->shift_y;
    h.shift_x = d->shift_x;
  }
  cx_fft_plane f{};
  f.pre_re = 1.0;
  f.post_re = 1.0;
  f.dy_in = f.dx_in = f.dy_out = f.dx_out = 1.0;
  f.pupil_r2 = -1.0;
  k_czt_prop_tables<<<1, 32, 0, st>>>(hp, h, fp, f);
  CX_LAUNCH_CHECK();
  cx_prop2d_desc hd{};
  hd.ny = L.py;
  hd.nx = L.px;
  hd.n_wv = 1;
  hd.n_in_planes = 1;
  hd.n_out_planes = 1;
  hd.kernel = d->kernel;
  hd.precision = d->precision;
  hd.remove_evanescent = d->kernel == CX_KERNEL_ASM ? d->remove_evanescent : 0;
  hd.bandlimit = d->bandlimit;
  hd.n_medium = d->n_medium;
  hd.ky0 = d->ky0;
  hd.kx0 = d->kx0;
  if ((s = cx_fill_propagator(&hd, hp, H, stream)) != CX_OK) return s;

  cx_optfft_desc od{};
  od.ny = d->ny;
  od.nx = d->nx;
  od.pad_y = d->pad_y;
  od.pad_x = d->pad_x;
  od.n_wv = 1;
  od.n_in_planes = 1;
  od.n_out_planes = 1;
  od.precision = d->precision;

  // CZT parameters per axis
  const double pi = 3.141592653589793238462643383279502884;
  const int m[2] = {d->my, d->mx};
  const int P[2] = {L.py, L.px};
  const double dxi[2] = {d->dy_in, d->dx_in};
  const double dxo[2] = {d->dy_out, d->dx_out};
  const double sh[2] = {d->shift_y, d->shift_x};
  std::complex<double> A[2], Wc[2];
  double alpha = 1.0;
  for (int k = 0; k < 2; ++k) {
    const double Tk = dxi[k] * P[k];
    alpha *= dxo[k] * Tk;
    const double lo = dxo[k] * (0.0 - m[k] / 2.0) + sh[k];
    const double hi = dxo[k] * ((m[k] - 1) - m[k] / 2.0) + sh[k];
    A[k] = std::exp(std::complex<double>(0.0, -2.0 * pi / Tk * lo));
    Wc[k] = std::exp(std::complex<double>(0.0, (2.0 * pi / Tk) * (hi - lo) / (m[k] - 1)));
  }

  const size_t in_plane = (size_t)d->ny * d->nx;
  const size_t out_plane = (size_t)d->my * d->mx;
  // Yu et al.: per axis n = padded length, alpha = dx_out / df_in with df_in =
  // 1 / (n dx_in); input factor (1/alpha) exp(i pi alpha df^2 (j - n//2)^2),
  // filter exp(-i pi alpha df^2 (m - n//2)^2) on m in [0, n) placed for the
  // "same" convolution (offset (n-1)//2), output factor
  // dx_out exp(i pi / alpha (dx_out (k - n/2) + origin)^2)
  CztArgs yu[2];
  if (d->method == 1) {
    const float2* twg = nullptr;
    if ((s = ensure_twiddles(&twg)) != CX_OK) return s;
    const int Ls[2] = {L.Ly, L.Lx};
    for (int k = 0; k < 2; ++k) {
      const int n = P[k];
      const double df = 1.0 / ((double)n * dxi[k]);
      const double al = dxo[k] / df;
      const double cin = al * df * df;
      const int sc = (n - 1) / 2;
      float2* cfilt = reinterpret_cast<float2*>(static_cast<char*>(cws)) + (size_t)k * 2 * (L.Ly > L.Lx ? L.Ly : L.Lx);
      float2* chat = cfilt + (L.Ly > L.Lx ? L.Ly : L.Lx);
      k_yu_filter<<<(Ls[k] + 255) / 256, 256, 0, st>>>(cfilt, Ls[k], cin, (double)(n - 1 - sc + n / 2), n - 1 - sc,
                                                       2 * n - 1 - sc);
      CX_LAUNCH_CHECK();
      if ((s = cx_fft1d(cfilt, chat, Ls[k], 1, 0, stream)) != CX_OK) return s;
      CztArgs& a = yu[k];
      a.n = n;
      a.m = n;
      a.L = Ls[k];
      a.ta = a.tw = a.la = a.lw = 0.0;
      a.modN = -1;
      a.scale = 1.0;
      a.chat = chat;
      a.twg = twg;
      a.kind = 1;
      a.c_in = cin;
      a.j0_in = (double)(n / 2);
      a.mag_in = 1.0 / al;
      a.c_out = 1.0 / al;
      a.dx_out = dxo[k];
      a.k0_out = n / 2.0;
      a.org_out = sh[k];
      a.mag_out = dxo[k];
    }
    // along y: column tiles over the px columns; along x: one team per row
    yu[0].n_vec = L.px;
    yu[0].inner = L.px;
    yu[0].in_ostride = (long)L.py * L.px;
    yu[0].in_istride = 1;
    yu[0].in_estride = L.px;
    yu[0].out_ostride = (long)L.py * L.px;
    yu[0].out_istride = 1;
    yu[0].out_estride = L.px;
    yu[1].n_vec = L.py;
    yu[1].inner = 1;
    yu[1].in_ostride = L.px;
    yu[1].in_istride = 1;
    yu[1].in_estride = 1;
    yu[1].out_ostride = L.px;
    yu[1].out_istride = 1;
    yu[1].out_estride = 1;
  }
  for (int b = 0; b < d->n_fields; ++b) {
    const float2* ub = static_cast<const float2*>(u_in) + (size_t)b * in_plane;
    float2* ob = static_cast<float2*>(u_out) + (size_t)b * out_plane;
    // Y = fftshift(H fft2(ifftshift(pad u))), with the optical FFT's own
    // workspace in T
    if ((s = cx_optical_fft_h(&od, fp, H, ub, Y, T, sizeof(float2) * (size_t)L.py * L.px, stream)) != CX_OK)
      return s;
    if (d->method == 1) {
      yu[0].x = Y;
      yu[0].y = T;
      if ((s = czt_dispatch_cols(yu[0].L, yu[0], st)) != CX_OK) return s;
      yu[1].x = T;
      yu[1].y = ob;
      if ((s = czt_dispatch_rows(yu[1].L, yu[1], st)) != CX_OK) return s;
      continue;
    }
    // along y: (py, px) -> (my, px), column tiles
    cx_czt_desc cy{};
    cy.n = L.py;
    cy.m = d->my;
    cy.L = L.Ly;
    cy.inner = L.px;
    cy.n_vec = L.px;
    cy.in_ostride = (int64_t)L.py * L.px;
    cy.in_istride = 1;
    cy.in_estride = L.px;
    cy.out_ostride = (int64_t)d->my * L.px;
    cy.out_istride = 1;
    cy.out_estride = L.px;
    cy.a_re = A[0].real();
    cy.a_im = A[0].imag();
    cy.w_re = Wc[0].real();
    cy.w_im = Wc[0].imag();
    cy.mod_n = (d->my - 1) / 2;
    cy.layout = 1;
    cy.scale = 1.0;
    if ((s = cx_czt(&cy, Y, T, cws, cws_bytes, stream)) != CX_OK) return s;
    // along x: (my, px) -> (my, mx), one team per row
    cx_czt_desc cxd{};
    cxd.n = L.px;
    cxd.m = d->mx;
    cxd.L = L.Lx;
    cxd.inner = 1;
    cxd.n_vec = d->my;
    cxd.in_ostride = L.px;
    cxd.in_istride = 1;
    cxd.in_estride = 1;
    cxd.out_ostride = d->mx;
    cxd.out_istride = 1;
    cxd.out_estride = 1;
    cxd.a_re = A[1].real();
    cxd.a_im = A[1].imag();
    cxd.w_re = Wc[1].real();
    cxd.w_im = Wc[1].imag();
    cxd.mod_n = (d->mx - 1) / 2;
    cxd.layout = 0;
    cxd.scale = 1.0 / alpha;
    if ((s = cx_czt(&cxd, T, ob, cws, cws_bytes, stream)) != CX_OK) return s;
  }
  return CX_OK;
}
