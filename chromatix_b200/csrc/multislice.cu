// C API of the multislice forward / adjoint (kernels in multislice.cuh and
// the prop2d column pass).
#include <cmath>
#include <mutex>

#include "multislice.cuh"

namespace cx {

struct MsPlan {
  int py, px, D, K, nseg;
  int last;  // slices of the last segment, whose records the forward keeps (no recomputation)
  Prop2DArgs col;  // column pass template (plane pointer set per launch)
};

// The slice propagator H(dz) is applied 2D times (and conj(H) D times in the
// adjoint): it is evaluated once per call into a table with FP64 sin/cos
// (correctly rounded to complex64), so its rounding does not accumulate
// across slices, and read back from L2 by every column pass.
__global__ void k_ms_fill_h(float2* __restrict__ H, Prop2DArgs a, cx_plane pl) {
  const long total = (long)a.py * a.px;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x)
    H[i] = prop_kernel(i / a.px, i % a.px, a, pl);
}

static cx_status ms_plan(const cx_ms_desc* d, MsPlan* p) {
  if (!d || d->ny <= 0 || d->nx <= 0 || d->pad < 0 || d->n_slices <= 0 || !(d->wavelength > 0.0) ||
      !(d->dy > 0.0) || !(d->dx > 0.0) || d->precision < 0 || d->precision > 2) {
    set_error("invalid multislice descriptor");
    return CX_ERR_INVALID;
  }
  p->py = d->ny + 2 * d->pad;
  p->px = d->nx + 2 * d->pad;
  if (!size_supported(p->py) || !size_supported(p->px)) {
    set_error("padded grid %dx%d: FFT length not supported", p->py, p->px);
    return CX_ERR_UNSUPPORTED;
  }
  if (d->precision == CX_PREC_SPLIT16 && !prop_tc_supported(p->py, p->px)) {
    set_error("CX_PREC_SPLIT16 multislice: padded grid %dx%d not compiled in (1024 or 1280 rows, columns a "
              "multiple of 8)", p->py, p->px);
    return CX_ERR_UNSUPPORTED;
  }
  p->D = d->n_slices;
  int K = d->checkpoint_every;
  if (K <= 0) K = (int)std::ceil(std::sqrt((double)p->D));
  if (K > p->D) K = p->D;
  p->K = K;
  p->nseg = (p->D + K - 1) / K;
  p->last = p->D - (p->nseg - 1) * K;
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
  a.precision = d->precision;
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
  return ensure_twiddles(&a.twg);
}

static size_t al(size_t b) { return (b + 255) & ~(size_t)255; }

// workspace: [planes (4 x cx_plane)] [H table] [F state] ([G state] [2 x K records] for the adjoint:
// the records of two segments, one being read by the adjoint while the next is recomputed)
static size_t ms_ws(const MsPlan& p, bool grad) {
  const size_t field = sizeof(float2) * (size_t)p.py * p.px;
  size_t b = al(4 * sizeof(cx_plane)) + 2 * al(field);
  if (grad) b += al(field) + 2 * (size_t)p.K * al(field);
  return b;
}

// Second stream of a device for the adjoint's recomputation chain (created
// once, non-blocking; ordered against the caller's stream by events only).
// nullptr if it cannot be created: the adjoint then runs on one stream.
static cudaStream_t ms_side_stream() {
  static std::mutex mu;
  static cudaStream_t side[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(mu);
  if (!side[dev] && cudaStreamCreateWithFlags(&side[dev], cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    side[dev] = nullptr;
  }
  return side[dev];
}

static MsArgs ms_args(const cx_ms_desc* d, const MsPlan& p) {
  MsArgs a{};
  a.ny = d->ny;
  a.nx = d->nx;
  a.pad_y = d->pad;
  a.pad_x = d->pad;
  a.py = p.py;
  a.px = p.px;
  a.precision = d->precision;
  a.lam = d->wavelength;
  a.dz = d->dz;
  a.kdz_f = (float)(6.283185307179586476925286766559 * d->dz / d->wavelength);
  a.twg = p.col.twg;
  a.load_scale = 1.f;
  return a;
}

// planes: 0 slice (+dz), 1 slice adjoint (-dz), 2 defocus (-dist), 3 defocus adjoint (+dist)
static cx_status ms_upload_planes(const cx_ms_desc* d, const MsPlan& p, cx_plane* dev, cudaStream_t st) {
  cx_plane h[4];
  const double zs[4] = {d->dz, -d->dz, -d->reverse_distance, d->reverse_distance};
  for (int i = 0; i < 4; ++i) {
    cx_plane& q = h[i];
    q = cx_plane{};
    q.z = zs[i];
    q.wavelength = d->wavelength;
    q.dy = d->dy;
    q.dx = d->dx;
    q.in_plane = 0;
    q.h_plane = 0;
    // Matsushima band limit for the slice propagator (propagation.py:557-579, shift 0)
    if (d->bandlimit && i < 2) {
      const double ext[2] = {d->dy * p.py, d->dx * p.px};
      double k0[2], km[2];
      for (int a = 0; a < 2; ++a) {
        const double df = 1.0 / ext[a];
        const double klp = std::pow(std::pow(1.0 / (2 * df), -2.0) * q.z * q.z + 1.0, -0.5) / d->wavelength;
        const double kln = std::pow(std::pow(-1.0 / (2 * df), -2.0) * q.z * q.z + 1.0, -0.5) / d->wavelength;
        k0[a] = 0.5 * (klp - kln);
        km[a] = (klp + kln) / 2.0;
      }
      q.bl_y0 = k0[0];
      q.bl_x0 = k0[1];
      q.bl_hy = km[0];
      q.bl_hx = km[1];
    }
  }
  CX_CUDA_TRY(cudaMemcpyAsync(dev, h, sizeof(h), cudaMemcpyHostToDevice, st));
  return CX_OK;
}

// slice_prop: the per-slice propagator, read from the H table (conjugated for
// the adjoint); otherwise the plain ASM defocus kernel evaluated on the fly
// (samples.py:268-270)
static cx_status col_pass(const MsPlan& p, const cx_plane* plane, float2* buf, double na_f2, bool slice_prop,
                          cudaStream_t st, const float2* Htab = nullptr, bool conj_h = false) {
  Prop2DArgs a = p.col;
  a.planes = plane;
  a.na_f2 = na_f2;
  if (slice_prop) {
    a.kernel = CX_KERNEL_EXPLICIT;
    a.H = Htab;
    a.conj_h = conj_h ? 1 : 0;
  } else {
    a.bandlimit = 0;
    a.remove_evanescent = 0;
  }
  return prop_cols(p.py, buf, buf, a, st);
}

static cx_status fill_h(const cx_ms_desc* d, const MsPlan& p, float2* H, cudaStream_t st) {
  Prop2DArgs a = p.col;
  a.precise = 1;
  cx_plane pl = cx_plane{};
  pl.z = d->dz;
  pl.wavelength = d->wavelength;
  pl.dy = d->dy;
  pl.dx = d->dx;
  if (d->bandlimit) {
    // Matsushima band limit, shift 0 (propagation.py:557-579): centre 0, half width k
    const double ext[2] = {d->dy * p.py, d->dx * p.px};
    double km[2];
    for (int i = 0; i < 2; ++i) {
      const double half_period = ext[i] / 2.0;  // 1 / (2 df)
      km[i] = std::pow(std::pow(half_period, -2.0) * pl.z * pl.z + 1.0, -0.5) / d->wavelength;
    }
    pl.bl_hy = km[0];
    pl.bl_hx = km[1];
  }
  long total = (long)p.py * p.px;
  int grid = (int)((total + 255) / 256);
  if (grid > sm_count() * 8) grid = sm_count() * 8;
  k_ms_fill_h<<<grid, 256, 0, st>>>(H, a, pl);
  CX_LAUNCH_CHECK();
  return CX_OK;
}

static double na_mask(const cx_ms_desc* d) {
  if (!(d->NA > 0.0)) return -1.0;
  const double r = d->NA / d->wavelength;
  return r * r;
}

}  // namespace cx

using namespace cx;

extern "C" cx_status cx_multislice_workspace_size(const cx_ms_desc* d, int32_t need_grad, size_t* bytes) {
  MsPlan p;
  cx_status s = ms_plan(d, &p);
  if (s != CX_OK) return s;
  if (!bytes) return CX_ERR_INVALID;
  *bytes = ms_ws(p, need_grad != 0);
  return CX_OK;
}

extern "C" int32_t cx_multislice_num_checkpoints(const cx_ms_desc* d) {
  MsPlan p;
  if (ms_plan(d, &p) != CX_OK) return -1;
  return p.nseg + p.last;
}

extern "C" cx_status cx_multislice_forward(const cx_ms_desc* d, const void* u_in, const float* dn, const float* ab,
                                           void* u_out, void* checkpoints, void* workspace, size_t workspace_bytes,
                                           cx_stream_t stream) {
  MsPlan p;
  cx_status s = ms_plan(d, &p);
  if (s != CX_OK) return s;
  if (!u_in || !dn || !ab || !u_out || !workspace) {
    set_error("null pointer argument");
    return CX_ERR_INVALID;
  }
  if (workspace_bytes < ms_ws(p, false)) {
    set_error("workspace too small: %zu < %zu", workspace_bytes, ms_ws(p, false));
    return CX_ERR_WORKSPACE;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  char* w = static_cast<char*>(workspace);
  const size_t field = (size_t)p.py * p.px;
  cx_plane* planes = reinterpret_cast<cx_plane*>(w);
  float2* Htab = reinterpret_cast<float2*>(w + al(4 * sizeof(cx_plane)));
  float2* F = reinterpret_cast<float2*>(w + al(4 * sizeof(cx_plane)) + al(sizeof(float2) * field));
  float2* ck = static_cast<float2*>(checkpoints);
  if ((s = ms_upload_planes(d, p, planes, st)) != CX_OK) return s;
  if ((s = fill_h(d, p, Htab, st)) != CX_OK) return s;
  MsArgs a = ms_args(d, p);
  a.dn = dn;
  a.ab = ab;
  a.buf = F;
  // u_0 = pad(u_in) -> FFT_x (recorded as checkpoint 0)
  a.mode = MS_LOAD;
  a.src = static_cast<const float2*>(u_in);
  a.sy = d->ny;
  a.sx = d->nx;
  a.oy = d->pad;
  a.ox = d->pad;
  a.record = ck ? 1 : 0;
  a.rec = ck;
  if ((s = ms_rows(a, st)) != CX_OK) return s;
  if ((s = col_pass(p, planes + 0, F, -1.0, true, st, Htab)) != CX_OK) return s;
  // checkpoints: u_0, u_K, u_2K, ... (nseg planes), then u_{i0+1} .. u_D of the
  // last segment (i0 = (nseg - 1) K), which the adjoint reads without recomputing
  a.mode = MS_FWD;
  const int i0_last = (p.nseg - 1) * p.K;
  for (int i = 1; i <= p.D; ++i) {
    a.slice = i - 1;  // u_i = t_{i-1} P(u_{i-1})
    a.record = 0;
    a.rec = nullptr;
    if (ck && i < p.D && i % p.K == 0) {
      a.record = 1;
      a.rec = ck + (size_t)(i / p.K) * field;
    } else if (ck && i > i0_last) {
      a.record = 1;
      a.rec = ck + (size_t)(p.nseg + i - i0_last - 1) * field;
    }
    if ((s = ms_rows(a, st)) != CX_OK) return s;
    if (i < p.D && (s = col_pass(p, planes + 0, F, -1.0, true, st, Htab)) != CX_OK) return s;
  }
  // defocus back to the chosen plane, NA mask, crop (samples.py:265-282)
  if ((s = col_pass(p, planes + 2, F, na_mask(d), false, st)) != CX_OK) return s;
  a.mode = MS_FINAL;
  a.record = 0;
  a.dst = static_cast<float2*>(u_out);
  return ms_rows(a, st);
}

extern "C" cx_status cx_multislice_backward(const cx_ms_desc* d, const float* dn, const float* ab,
                                            const void* checkpoints, const void* grad_out, float* grad_dn,
                                            float* grad_ab, void* grad_u_in, void* workspace, size_t workspace_bytes,
                                            cx_stream_t stream) {
  MsPlan p;
  cx_status s = ms_plan(d, &p);
  if (s != CX_OK) return s;
  if (!dn || !ab || !checkpoints || !grad_out || !grad_dn || !grad_ab || !workspace) {
    set_error("null pointer argument");
    return CX_ERR_INVALID;
  }
  if (workspace_bytes < ms_ws(p, true)) {
    set_error("workspace too small: %zu < %zu", workspace_bytes, ms_ws(p, true));
    return CX_ERR_WORKSPACE;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const size_t field = (size_t)p.py * p.px;
  char* w = static_cast<char*>(workspace);
  cx_plane* planes = reinterpret_cast<cx_plane*>(w);
  w += al(4 * sizeof(cx_plane));
  float2* Htab = reinterpret_cast<float2*>(w);
  w += al(sizeof(float2) * field);
  float2* F = reinterpret_cast<float2*>(w);
  w += al(sizeof(float2) * field);
  float2* G = reinterpret_cast<float2*>(w);
  w += al(sizeof(float2) * field);
  float2* seg = reinterpret_cast<float2*>(w);
  const size_t seg_stride = al(sizeof(float2) * field) / sizeof(float2);
  const float2* ck = static_cast<const float2*>(checkpoints);
  if ((s = ms_upload_planes(d, p, planes, st)) != CX_OK) return s;
  if ((s = fill_h(d, p, Htab, st)) != CX_OK) return s;

  MsArgs g = ms_args(d, p);
  g.dn = dn;
  g.ab = ab;
  g.buf = G;
  // g_D = Q^H pad(g_out)
  g.mode = MS_LOAD;
  g.src = static_cast<const float2*>(grad_out);
  g.sy = d->ny;
  g.sx = d->nx;
  g.oy = d->pad;
  g.ox = d->pad;
  g.record = 0;
  if ((s = ms_rows(g, st)) != CX_OK) return s;
  if ((s = col_pass(p, planes + 3, G, na_mask(d), false, st)) != CX_OK) return s;

  // Segment sgi (slices i0 .. i1-1): the adjoint through slices i1-1 .. i0
  // reads u_{i0+1} .. u_{i1}.  The last segment's were recorded by the
  // forward (after the nseg checkpoints); every other segment's are
  // recomputed from its checkpoint u_{i0} into records[sgi & 1].  The
  // recomputation of segment sgi - 1 needs only its checkpoint, so it runs on
  // a second stream (rs) while the adjoint works through segment sgi (one pass
  // alone fills few SMs: a 1024^2 plane is 1024 transforms).  Order:
  // adjoint(sgi) waits for recompute(sgi); recompute(sgi - 2), which
  // overwrites the same record half, waits for adjoint(sgi) (the last
  // segment reads no half, so recompute(nseg - 3) starts at once).  Both
  // chains run the same kernels on the same data as a serial run, so the
  // gradients are the same bits.
  MsArgs f = ms_args(d, p);
  f.dn = dn;
  f.ab = ab;
  f.buf = F;
  auto recompute = [&](int sgi, cudaStream_t q) -> cx_status {
    const int i0 = sgi * p.K, i1 = (i0 + p.K < p.D) ? i0 + p.K : p.D;
    float2* recs = seg + (size_t)(sgi & 1) * p.K * seg_stride;
    cx_status e;
    f.mode = MS_LOAD;
    f.src = ck + (size_t)sgi * field;
    f.sy = p.py;
    f.sx = p.px;
    f.oy = 0;
    f.ox = 0;
    f.record = 0;
    if ((e = ms_rows(f, q)) != CX_OK) return e;
    if ((e = col_pass(p, planes + 0, F, -1.0, true, q, Htab)) != CX_OK) return e;
    f.mode = MS_FWD;
    for (int i = i0 + 1; i <= i1; ++i) {
      f.slice = i - 1;
      f.record = 1;
      f.rec = recs + (size_t)(i - i0 - 1) * seg_stride;
      if ((e = ms_rows(f, q)) != CX_OK) return e;
      if (i < i1 && (e = col_pass(p, planes + 0, F, -1.0, true, q, Htab)) != CX_OK) return e;
    }
    return CX_OK;
  };
  auto adjoint = [&](int sgi, cudaStream_t q) -> cx_status {
    const int i0 = sgi * p.K, i1 = (i0 + p.K < p.D) ? i0 + p.K : p.D;
    const bool last = sgi == p.nseg - 1;
    const float2* recs = last ? ck + (size_t)p.nseg * field : seg + (size_t)(sgi & 1) * p.K * seg_stride;
    const size_t stride = last ? field : seg_stride;
    cx_status e;
    g.mode = MS_BWD;
    for (int i = i1 - 1; i >= i0; --i) {
      g.slice = i;
      g.rec_u = recs + (size_t)(i - i0) * stride;
      g.gdn = grad_dn + (size_t)i * d->ny * d->nx;
      g.gab = grad_ab + (size_t)i * d->ny * d->nx;
      if ((e = ms_rows(g, q)) != CX_OK) return e;
      if ((e = col_pass(p, planes + 1, G, -1.0, true, q, Htab, true)) != CX_OK) return e;
    }
    return CX_OK;
  };

  cudaStream_t rs = ms_side_stream();
  cudaEvent_t ev[4] = {};  // fork, recomputed (two halves), adjoint done
  int made = 0;
  if (rs && rs != st) {
    for (; made < 4; ++made)
      if (cudaEventCreateWithFlags(&ev[made], cudaEventDisableTiming) != cudaSuccess) break;
    if (made < 4) {
      cudaGetLastError();
      rs = nullptr;
    }
  } else {
    rs = nullptr;
  }
  cudaError_t ce = cudaSuccess;
  if (rs) {
    // the recomputation reads the checkpoints, the H table and the planes written on st
    if ((ce = cudaEventRecord(ev[0], st)) == cudaSuccess) ce = cudaStreamWaitEvent(rs, ev[0], 0);
  }
  s = CX_OK;
  if (rs) {
    for (int t = p.nseg - 2; t >= 0 && t >= p.nseg - 3 && ce == cudaSuccess && s == CX_OK; --t)
      if ((s = recompute(t, rs)) == CX_OK) ce = cudaEventRecord(ev[1 + (t & 1)], rs);
  }
  for (int sgi = p.nseg - 1; sgi >= 0 && ce == cudaSuccess && s == CX_OK; --sgi) {
    if (sgi < p.nseg - 1) {
      if (rs && (ce = cudaStreamWaitEvent(st, ev[1 + (sgi & 1)], 0)) != cudaSuccess) break;
      if (!rs && (s = recompute(sgi, st)) != CX_OK) break;
    }
    if ((s = adjoint(sgi, st)) != CX_OK) break;
    if (rs && sgi >= 2 && sgi <= p.nseg - 2) {
      if ((ce = cudaEventRecord(ev[3], st)) != cudaSuccess) break;
      if ((ce = cudaStreamWaitEvent(rs, ev[3], 0)) != cudaSuccess) break;
      if ((s = recompute(sgi - 2, rs)) != CX_OK) break;
      ce = cudaEventRecord(ev[1 + (sgi & 1)], rs);
    }
  }
  if (rs && (s != CX_OK || ce != cudaSuccess)) {
    // failed part-way: st still takes up everything issued on rs
    if (cudaEventRecord(ev[0], rs) == cudaSuccess) cudaStreamWaitEvent(st, ev[0], 0);
  }
  for (int k = 0; k < made; ++k) cudaEventDestroy(ev[k]);
  if (s != CX_OK) return s;
  if (ce != cudaSuccess) {
    set_error("cx_multislice_backward: %s", cudaGetErrorString(ce));
    return CX_ERR_CUDA;
  }
  if (grad_u_in) {
    g.mode = MS_FINAL;
    g.dst = static_cast<float2*>(grad_u_in);
    return ms_rows(g, st);
  }
  return CX_OK;
}
