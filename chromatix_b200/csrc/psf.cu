// C API of the fused batched 4f PSF (kernels in psf.cuh).
#include <cmath>
#include <cstdlib>

#include "psf.cuh"

namespace cx {

// ---------------------------------------------------------------------------
// pass 0: pupil pixel counts (one counter per wavelength, zeroed by the host)
// ---------------------------------------------------------------------------
// One thread per (wavelength, row): the pupil is a disc, so the pixels of a
// row that pass the (exact, per-pixel) pupil predicate form one contiguous
// run around the centre column; its ends are found by bisection with the
// same predicate the kernels use.  Also records the exact range of rows that
// hold pupil pixels: srange[w] = max(ny - y), srange[8 + w] = max(y + 1)
// (zero-initialised, so an empty pupil gives the empty range [ny, 0)).
__global__ void k_psf_count(PsfArgs a, unsigned long long* counts, int* srange) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.W * a.ny) return;
  const int w = i / a.ny, y = i % a.ny;
  const PsfWv& p = a.wv[w];
  const int xc = a.nx / 2;  // grid value 0 (x = nx/2): the widest point of the chord
  if (!in_pupil(a, p, y, xc)) return;
  // last inside column to the right of xc, first inside column to the left
  int lo = xc, hi = a.nx;  // in_pupil(lo) true, columns >= hi outside
  while (hi - lo > 1) {
    const int m = (lo + hi) / 2;
    if (in_pupil(a, p, y, m)) lo = m; else hi = m;
  }
  const int right = lo;
  lo = -1;
  hi = xc;  // columns <= lo outside, in_pupil(hi) true
  while (hi - lo > 1) {
    const int m = (lo + hi) / 2;
    if (in_pupil(a, p, y, m)) hi = m; else lo = m;
  }
  const int left = hi;
  atomicAdd(counts + w, (unsigned long long)(right - left + 1));
  atomicMax(srange + w, a.ny - y);
  atomicMax(srange + 8 + w, y + 1);
}

// ---------------------------------------------------------------------------
// accurate-mode source tables (PsfArgs::M, PsfArgs::CX), FP64 phases
// ---------------------------------------------------------------------------
__global__ void k_psf_tables(PsfArgs a) {
  const long ncx = (long)a.nz * a.csum;
  const double PI = 3.141592653589793238462643383279502884;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < a.msum + ncx; i += (long)gridDim.x * blockDim.x) {
    if (i < a.msum) {
      int w = 0;
      while (w + 1 < a.W && i >= a.mprefix[w + 1]) ++w;
      const PsfWv& p = a.wv[w];
      const long loc = i - a.mprefix[w];
      const int y = a.ylo[w] + (int)(loc / a.ncols[w]), x = a.xlo[w] + (int)(loc % a.ncols[w]);
      float2 v = make_float2(0.f, 0.f);
      if (y < a.ny && x < a.nx && in_pupil(a, p, y, x)) {
        v = psf_const(a, w, a.counts);
        if (a.has_phase) v = cmul(v, expi_precise((double)a.phase[(size_t)y * a.nx + x] * p.mod));
      }
      a.M[i] = v;
    } else {
      const long j = i - a.msum;
      const int iz = (int)(j / a.csum), loc = (int)(j % a.csum);
      int w = 0;
      while (w + 1 < a.W && loc >= a.cprefix[w + 1]) ++w;
      const PsfWv& p = a.wv[w];
      const int x = a.xlo[w] + (loc - a.cprefix[w]);
      const double gxo = p.dx * ((double)x - (double)a.nx * 0.5) - a.offx;
      const double qz = -PI * (a.z[iz] / a.f_obj) / p.L2;
      a.CX[j] = expi_precise(qz * gxo * gxo);
    }
  }
}

// ---------------------------------------------------------------------------
// materialised source field (objective_point_source [-> phase_change]) for
// callers that need u itself: out (zc, ny, nx, W) complex64, without the lens
// normalisation
// ---------------------------------------------------------------------------
__global__ void k_psf_source(PsfArgs a, float2* __restrict__ out) {
  const long per = (long)a.ny * a.nx;
  const long total = per * a.nz * a.W;
  const double PI = 3.141592653589793238462643383279502884;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int w = (int)(i % a.W);
    const long pix = (i / a.W) % per;
    const int iz = (int)(i / ((long)a.W * per));
    const int y = (int)(pix / a.nx), x = (int)(pix % a.nx);
    const PsfWv& p = a.wv[w];
    float2 v = make_float2(0.f, 0.f);
    if (in_pupil(a, p, y, x)) {
      const float2 cst = psf_const(a, w, a.counts);
      const double z = a.z[iz];
      if (a.precision == CX_PREC_REF32) {
        const float gyf = fm((float)p.dy, (float)y - (float)a.ny * 0.5f);
        const float gxf = fm((float)p.dx, (float)x - (float)a.nx * 0.5f);
        const float dyo = fs(gyf, (float)a.offy), dxo = fs(gxf, (float)a.offx);
        const float r2 = fa(fm(dyo, dyo), fm(dxo, dxo));
        const float phs = fd(fm(fm(-3.14159265358979f, fd((float)z, (float)a.f_obj)), r2), p.L2f);
        float s1, c1;
        sincosf(phs, &s1, &c1);
        v = cmul(cst, make_float2(c1, s1));
        if (a.has_phase) {
          float s2, c2;
          sincosf(fm(a.phase[pix], p.modf), &s2, &c2);
          v = cmul(v, make_float2(c2, s2));
        }
      } else {
        const double gyo = p.dy * ((double)y - (double)a.ny * 0.5) - a.offy;
        const double gxo = p.dx * ((double)x - (double)a.nx * 0.5) - a.offx;
        double ph = -PI * (z / a.f_obj) / p.L2 * (gyo * gyo + gxo * gxo);
        if (a.has_phase) ph += (double)a.phase[pix] * p.mod;
        v = cmul(cst, expi_reduced(ph));
      }
    }
    out[i] = v;
  }
}

// rows of the grid that can hold pupil pixels for wavelength w (a
// conservative superset, one row of margin: the kernels re-test every row)
static void psf_rows(const cx_psf_desc* d, const cx_psf_spectrum* spec, int w, int* ylo, int* nrows) {
  const double lam0 = spec->wavelength[0];
  const double D = 2.0 * d->f_obj * d->NA / d->n_medium;
  double r = (lam0 / spec->wavelength[w]) * D / 2.0;
  if (d->lens_NA > 0.0) {
    const double rl = (lam0 / spec->wavelength[w]) * (2.0 * d->f_lens * d->lens_NA / d->n_medium) / 2.0;
    r = rl < r ? rl : r;
  }
  const double h = r / spec->dy[w];
  long lo = (long)floor(0.5 * d->ny - h) - 1, hi = (long)ceil(0.5 * d->ny + h) + 1;
  if (lo < 0) lo = 0;
  if (hi > d->ny - 1) hi = d->ny - 1;
  if (hi < lo) hi = lo;
  *ylo = (int)lo;
  *nrows = (int)(hi - lo + 1);
}

// columns of the grid that can hold pupil pixels for wavelength w (same
// conservative rule as psf_rows, along x)
static void psf_cols_box(const cx_psf_desc* d, const cx_psf_spectrum* spec, int w, int* xlo, int* ncols) {
  const double lam0 = spec->wavelength[0];
  const double D = 2.0 * d->f_obj * d->NA / d->n_medium;
  double r = (lam0 / spec->wavelength[w]) * D / 2.0;
  if (d->lens_NA > 0.0) {
    const double rl = (lam0 / spec->wavelength[w]) * (2.0 * d->f_lens * d->lens_NA / d->n_medium) / 2.0;
    r = rl < r ? rl : r;
  }
  const double h = r / spec->dx[w];
  long lo = (long)floor(0.5 * d->nx - h) - 1, hi = (long)ceil(0.5 * d->nx + h) + 1;
  if (lo < 0) lo = 0;
  if (hi > d->nx - 1) hi = d->nx - 1;
  if (hi < lo) hi = lo;
  *xlo = (int)lo;
  *ncols = (int)(hi - lo + 1);
}

// Row spectra of one z-chunk are written by pass A and read back by pass B;
// the chunk is sized to stay L2-resident in between (CX_PSF_L2_MB, default
// 64 MiB of the 126 MB L2).
static size_t psf_chunk_budget() {
  static size_t cached = 0;
  if (!cached) {
    const char* e = getenv("CX_PSF_L2_MB");
    const long mb = e ? atol(e) : 64;
    cached = (size_t)(mb > 0 ? mb : 64) << 20;
  }
  return cached;
}

static cx_status psf_check(const cx_psf_desc* d) {
  if (!d || d->ny <= 0 || d->nx <= 0 || d->n_z <= 0 || d->n_wv <= 0 || d->n_wv > PSF_MAX_WV) {
    set_error("invalid PSF descriptor (1 <= n_wv <= %d)", PSF_MAX_WV);
    return CX_ERR_INVALID;
  }
  if (!size_supported(d->ny) || !size_supported(d->nx)) {
    set_error("PSF grid %dx%d: FFT length not supported", d->ny, d->nx);
    return CX_ERR_UNSUPPORTED;
  }
  if (!(d->f_lens > 0.0)) {
    set_error("cx_psf_4f needs a forward lens (f_lens > 0); use cx_optical_fft for inverse lenses");
    return CX_ERR_INVALID;
  }
  if (d->precision < 0 || d->precision > 2) {
    set_error("invalid PSF precision %d", d->precision);
    return CX_ERR_INVALID;
  }
  if (d->precision == CX_PREC_SPLIT16 && !psf_tc_supported(d->ny, d->nx)) {
    set_error("CX_PREC_SPLIT16 PSF: grid %dx%d not compiled in (ny 1024 or 1280, nx a multiple of 8)", d->ny,
              d->nx);
    return CX_ERR_UNSUPPORTED;
  }
  return CX_OK;
}

static PsfArgs psf_make_args(const cx_psf_desc* d, const cx_psf_spectrum* spec, bool with_lens) {
  PsfArgs a{};
  a.ny = d->ny;
  a.nx = d->nx;
  a.nz = d->n_z;
  a.W = d->n_wv;
  a.precision = d->precision;
  a.has_phase = d->has_phase;
  a.normalize = d->normalize_power;
  a.f_obj = d->f_obj;
  a.n = d->n_medium;
  a.amp = d->amplitude;
  a.offy = d->offset_y;
  a.offx = d->offset_x;
  a.power = d->power;
  const double lam0 = spec->wavelength[0];
  const double D = 2.0 * d->f_obj * d->NA / d->n_medium;                                   // sources.py:205
  const double DL = d->lens_NA > 0.0 ? 2.0 * d->f_lens * d->lens_NA / d->n_medium : -1.0;  // lenses.py:90
  for (int w = 0; w < a.W; ++w) {
    PsfWv& p = a.wv[w];
    p.lam = spec->wavelength[w];
    p.dens = spec->density[w];
    p.dy = spec->dy[w];
    p.dx = spec->dx[w];
    p.L2 = p.lam * d->f_obj / d->n_medium;
    const double r = (lam0 / p.lam) * D / 2.0;
    p.R2 = r * r;
    const double rl = (lam0 / p.lam) * DL / 2.0;
    p.RL2 = DL > 0.0 ? rl * rl : -1.0;
    p.mod = d->spectrally_modulate ? lam0 / p.lam : 1.0;
    // optical_fft forward normalisation -1j * dy dx / L_sq, L_sq = lam f / n (convenience.py:33,43)
    if (with_lens) {
      const double Lsq = p.lam * d->f_lens / d->n_medium;
      p.lens_re = 0.0;
      p.lens_im = -(p.dy * p.dx) / Lsq;
    } else {
      p.lens_re = 1.0;
      p.lens_im = 0.0;
    }
    // float32 reference-order values
    const float Lf = sqrtf((float)p.lam * (float)d->f_obj / (float)d->n_medium);
    p.L2f = Lf * Lf;
    const float rf = (float)lam0 / (float)p.lam * (float)D / 2.0f;
    p.R2f = rf * rf;
    const float rlf = (float)lam0 / (float)p.lam * (float)DL / 2.0f;
    p.RL2f = DL > 0.0 ? rlf * rlf : -1.0f;
    p.modf = (float)p.mod;
  }
  return a;
}

// workspace: 256 bytes of pupil counters, then one chunk of row spectra
// (sized for the worst case rowsum = n_wv * ny, independent of the spectrum)
static size_t psf_t_bytes(const cx_psf_desc* d) {
  const size_t worst_z = (size_t)d->n_wv * d->ny * d->nx * sizeof(float2);
  const size_t t = psf_chunk_budget() > worst_z ? psf_chunk_budget() : worst_z;
  return (t + 255) & ~(size_t)255;
}
static size_t psf_m_bytes(const cx_psf_desc* d) {
  return ((size_t)d->n_wv * d->ny * d->nx * sizeof(float2) + 255) & ~(size_t)255;
}
static size_t psf_ws(const cx_psf_desc* d) {
  const size_t cx_bytes = ((size_t)d->n_z * d->n_wv * d->nx * sizeof(float2) + 255) & ~(size_t)255;
  return 256 + psf_t_bytes(d) + psf_m_bytes(d) + cx_bytes;
}

}  // namespace cx

using namespace cx;

extern "C" cx_status cx_psf_workspace_size(const cx_psf_desc* d, size_t* bytes) {
  cx_status s = psf_check(d);
  if (s != CX_OK) return s;
  if (!bytes) return CX_ERR_INVALID;
  *bytes = psf_ws(d);
  return CX_OK;
}

namespace cx {

// shared set-up of cx_psf_4f / cx_psf_4f_stage: arguments, compact-row
// geometry and the z-chunk size
static cx_status psf_setup(const cx_psf_desc* d, const cx_psf_spectrum* spec, const double* z_dev, const float* phase,
                           float* intensity_out, void* workspace, size_t workspace_bytes, PsfArgs* out_args,
                           int* zc_out) {
  cx_status s = psf_check(d);
  if (s != CX_OK) return s;
  if (!spec || !spec->wavelength || !spec->density || !spec->dy || !spec->dx || !z_dev || !intensity_out ||
      !workspace || (d->has_phase && !phase)) {
    set_error("null pointer argument");
    return CX_ERR_INVALID;
  }
  if (workspace_bytes < psf_ws(d)) {
    set_error("workspace too small: %zu < %zu", workspace_bytes, psf_ws(d));
    return CX_ERR_WORKSPACE;
  }
  PsfArgs a = psf_make_args(d, spec, /*with_lens=*/true);
  a.z = z_dev;
  a.phase = phase;
  a.out = intensity_out;
  a.counts = static_cast<unsigned long long*>(workspace);
  a.srange = reinterpret_cast<int*>(static_cast<char*>(workspace) + 64);
  a.T = reinterpret_cast<float2*>(static_cast<char*>(workspace) + 256);
  if ((s = ensure_twiddles(&a.twg)) != CX_OK) return s;
  a.rowsum = 0;
  a.msum = 0;
  a.csum = 0;
  for (int w = 0; w < a.W; ++w) {
    psf_rows(d, spec, w, &a.ylo[w], &a.nrows[w]);
    a.prefix[w] = a.rowsum;
    a.rowsum += a.nrows[w];
    psf_cols_box(d, spec, w, &a.xlo[w], &a.ncols[w]);
    a.mprefix[w] = (int)a.msum;
    a.msum += (long)a.nrows[w] * a.ncols[w];
    a.cprefix[w] = a.csum;
    a.csum += a.ncols[w];
  }
  a.M = reinterpret_cast<float2*>(static_cast<char*>(workspace) + 256 + psf_t_bytes(d));
  a.CX = reinterpret_cast<float2*>(static_cast<char*>(workspace) + 256 + psf_t_bytes(d) + psf_m_bytes(d));
  // z planes per chunk: as many compact planes as the row-spectrum region holds
  const size_t zbytes = sizeof(float2) * (size_t)a.rowsum * a.nx;
  int zc = (int)(psf_t_bytes(d) / zbytes);
  if (zc < 1) zc = 1;
  if (zc > a.nz) zc = a.nz;
  *out_args = a;
  *zc_out = zc;
  return CX_OK;
}

static cx_status psf_prepare(const PsfArgs& a, void* workspace, cudaStream_t st) {
  CX_CUDA_TRY(cudaMemsetAsync(workspace, 0, 256, st));
  k_psf_count<<<(a.W * a.ny + 127) / 128, 128, 0, st>>>(a, const_cast<unsigned long long*>(a.counts),
                                                         const_cast<int*>(a.srange));
  CX_LAUNCH_CHECK();
  if (a.precision != CX_PREC_REF32) {
    const long n = a.msum + (long)a.nz * a.csum;
    const int blocks = (int)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096);
    k_psf_tables<<<blocks, 256, 0, st>>>(a);
    CX_LAUNCH_CHECK();
  }
  return CX_OK;
}

}  // namespace cx

using namespace cx;

extern "C" cx_status cx_psf_4f(const cx_psf_desc* d, const cx_psf_spectrum* spec, const double* z_dev,
                               const float* phase, float* intensity_out, void* workspace, size_t workspace_bytes,
                               cx_stream_t stream) {
  PsfArgs a;
  int zc = 1;
  cx_status s = psf_setup(d, spec, z_dev, phase, intensity_out, workspace, workspace_bytes, &a, &zc);
  if (s != CX_OK) return s;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if ((s = psf_prepare(a, workspace, st)) != CX_OK) return s;
  for (int z0 = 0; z0 < a.nz; z0 += zc) {
    a.z0 = z0;
    a.zc = (a.nz - z0) < zc ? (a.nz - z0) : zc;
    if ((s = psf_rows_pass(a, st)) != CX_OK) return s;
    if ((s = psf_cols(a, st)) != CX_OK) return s;
  }
  return CX_OK;
}

extern "C" cx_status cx_psf_plan_info(const cx_psf_desc* d, const cx_psf_spectrum* spec, int32_t* info) {
  if (!info) return CX_ERR_INVALID;
  cx_status s = psf_check(d);
  if (s != CX_OK) return s;
  int rowsum = 0;
  for (int w = 0; w < d->n_wv; ++w) {
    int lo, nr;
    psf_rows(d, spec, w, &lo, &nr);
    rowsum += nr;
  }
  const size_t zbytes = sizeof(float2) * (size_t)rowsum * d->nx;
  int zc = (int)(psf_t_bytes(d) / zbytes);
  if (zc < 1) zc = 1;
  if (zc > d->n_z) zc = d->n_z;
  info[0] = zc;
  info[1] = rowsum;
  info[2] = (d->n_z + zc - 1) / zc;
  info[3] = 0;
  return CX_OK;
}

extern "C" cx_status cx_psf_4f_stage(const cx_psf_desc* d, const cx_psf_spectrum* spec, const double* z_dev,
                                     const float* phase, float* intensity_out, void* workspace,
                                     size_t workspace_bytes, int32_t stage, int32_t chunk, cx_stream_t stream) {
  PsfArgs a;
  int zc = 1;
  cx_status s = psf_setup(d, spec, z_dev, phase, intensity_out, workspace, workspace_bytes, &a, &zc);
  if (s != CX_OK) return s;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (stage < 0) return psf_prepare(a, workspace, st);
  a.z0 = chunk * zc;
  if (a.z0 < 0 || a.z0 >= a.nz) {
    set_error("chunk %d out of range", chunk);
    return CX_ERR_INVALID;
  }
  a.zc = (a.nz - a.z0) < zc ? (a.nz - a.z0) : zc;
  return stage == 0 ? psf_rows_pass(a, st) : psf_cols(a, st);
}

// ---------------------------------------------------------------------------
// cx_psf_4f_to_host: the PSF stack streamed into host memory.  Groups of whole
// z-chunks are computed on `stream` into a ring of device slots; each group's
// device-to-host copy runs on `copy_stream` while the next groups compute.
// ---------------------------------------------------------------------------

namespace cx {

constexpr int kPsfHostSlots = 3;
constexpr int kPsfHostGroups = 8;  // target number of copy groups per stack

// group = z-planes per copy group; first = planes of the first group (one
// chunk, so that the first copy starts early)
static cx_status psf_host_plan(const cx_psf_desc* d, const cx_psf_spectrum* spec, int* group, size_t* slot_bytes,
                               int* first = nullptr) {
  int32_t info[4];
  cx_status s = cx_psf_plan_info(d, spec, info);
  if (s != CX_OK) return s;
  const int zc = info[0], chunks = info[2];
  const int per_group = (chunks + kPsfHostGroups - 1) / kPsfHostGroups;
  int g = zc * (per_group > 0 ? per_group : 1);
  if (g > d->n_z) g = d->n_z;
  *group = g;
  if (first) *first = zc < g ? zc : g;
  *slot_bytes = (((size_t)g * d->ny * d->nx * sizeof(float)) + 255) & ~(size_t)255;
  return CX_OK;
}

}  // namespace cx

extern "C" cx_status cx_psf_host_workspace_size(const cx_psf_desc* d, const cx_psf_spectrum* spec, size_t* bytes) {
  cx_status s = psf_check(d);
  if (s != CX_OK) return s;
  if (!bytes || !spec || !spec->wavelength || !spec->dy || !spec->dx) {
    set_error("null pointer argument");
    return CX_ERR_INVALID;
  }
  int g = 1;
  size_t slot = 0;
  if ((s = psf_host_plan(d, spec, &g, &slot)) != CX_OK) return s;
  cx_psf_desc dg = *d;
  dg.n_z = g;
  *bytes = psf_ws(&dg) + kPsfHostSlots * slot;
  return CX_OK;
}

extern "C" cx_status cx_psf_4f_to_host(const cx_psf_desc* d, const cx_psf_spectrum* spec, const double* z_dev,
                                       const float* phase, float* intensity_host, void* workspace,
                                       size_t workspace_bytes, cx_stream_t stream, cx_stream_t copy_stream) {
  cx_status s = psf_check(d);
  if (s != CX_OK) return s;
  if (!intensity_host || !workspace || !z_dev) {
    set_error("null pointer argument");
    return CX_ERR_INVALID;
  }
  size_t need = 0;
  if ((s = cx_psf_host_workspace_size(d, spec, &need)) != CX_OK) return s;
  if (workspace_bytes < need) {
    set_error("workspace too small: %zu < %zu", workspace_bytes, need);
    return CX_ERR_WORKSPACE;
  }
  int g = 1, g0 = 1;
  size_t slot = 0;
  if ((s = psf_host_plan(d, spec, &g, &slot, &g0)) != CX_OK) return s;
  cx_psf_desc dg = *d;
  dg.n_z = g;
  const size_t pws = psf_ws(&dg);
  char* ring = static_cast<char*>(workspace) + pws;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaStream_t cs = copy_stream ? static_cast<cudaStream_t>(copy_stream) : st;
  const size_t plane = (size_t)d->ny * d->nx;
  cudaEvent_t computed[kPsfHostSlots], copied[kPsfHostSlots];
  int made = 0;
  cudaError_t e = cudaSuccess;
  for (; made < kPsfHostSlots; ++made) {
    if ((e = cudaEventCreateWithFlags(&computed[made], cudaEventDisableTiming)) != cudaSuccess) break;
    if ((e = cudaEventCreateWithFlags(&copied[made], cudaEventDisableTiming)) != cudaSuccess) {
      cudaEventDestroy(computed[made]);
      break;
    }
  }
  if (e == cudaSuccess) {
    for (int z0 = 0, j = 0, gj = g0; z0 < d->n_z && s == CX_OK && e == cudaSuccess; z0 += gj, ++j, gj = g) {
      const int k = j % kPsfHostSlots;
      const int nz = (d->n_z - z0) < gj ? (d->n_z - z0) : gj;
      float* dst = reinterpret_cast<float*>(ring + (size_t)k * slot);
      if (j >= kPsfHostSlots && (e = cudaStreamWaitEvent(st, copied[k], 0)) != cudaSuccess) break;
      cx_psf_desc dj = *d;
      dj.n_z = nz;
      if ((s = cx_psf_4f(&dj, spec, z_dev + z0, phase, dst, workspace, pws, stream)) != CX_OK) break;
      if ((e = cudaEventRecord(computed[k], st)) != cudaSuccess) break;
      if ((e = cudaStreamWaitEvent(cs, computed[k], 0)) != cudaSuccess) break;
      if ((e = cudaMemcpyAsync(intensity_host + (size_t)z0 * plane, dst, sizeof(float) * nz * plane,
                               cudaMemcpyDeviceToHost, cs)) != cudaSuccess)
        break;
      if ((e = cudaEventRecord(copied[k], cs)) != cudaSuccess) break;
    }
    // the call is complete in `stream` order once the last copy is
    if (e == cudaSuccess && s == CX_OK && cs != st) {
      for (int k = 0; k < kPsfHostSlots && e == cudaSuccess; ++k) e = cudaStreamWaitEvent(st, copied[k], 0);
    }
  }
  for (int k = 0; k < made; ++k) {
    cudaEventDestroy(computed[k]);
    cudaEventDestroy(copied[k]);
  }
  if (s != CX_OK) return s;
  if (e != cudaSuccess) {
    set_error("cx_psf_4f_to_host: %s", cudaGetErrorString(e));
    return CX_ERR_CUDA;
  }
  return CX_OK;
}

extern "C" cx_status cx_psf_source(const cx_psf_desc* d, const cx_psf_spectrum* spec, const double* z_dev,
                                   const float* phase, void* u_out, void* workspace, size_t workspace_bytes,
                                   cx_stream_t stream) {
  if (!d || d->ny <= 0 || d->nx <= 0 || d->n_z <= 0 || d->n_wv <= 0 || d->n_wv > PSF_MAX_WV || !spec || !z_dev ||
      !u_out || !workspace || workspace_bytes < 256 || (d->has_phase && !phase)) {
    set_error("invalid point-source arguments");
    return CX_ERR_INVALID;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  PsfArgs a = psf_make_args(d, spec, /*with_lens=*/false);
  a.z = z_dev;
  a.phase = phase;
  unsigned long long* counts = static_cast<unsigned long long*>(workspace);
  int* srange = reinterpret_cast<int*>(static_cast<char*>(workspace) + 64);
  a.counts = counts;
  a.srange = srange;
  CX_CUDA_TRY(cudaMemsetAsync(workspace, 0, 256, st));
  k_psf_count<<<(a.W * a.ny + 127) / 128, 128, 0, st>>>(a, counts, srange);
  CX_LAUNCH_CHECK();
  k_psf_source<<<sm_count() * 8, 256, 0, st>>>(a, static_cast<float2*>(u_out));
  CX_LAUNCH_CHECK();
  return CX_OK;
}
