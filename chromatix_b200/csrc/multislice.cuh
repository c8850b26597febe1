// Thick-sample multislice: row passes of the forward and adjoint slice loop.
//
// Reference: functional/samples.py:137-282 (multislice_thick_sample) with
// thin_sample (samples.py:85-134) and the ASM kernel (propagation.py:499-580).
//
// The field state lives in one (py, px) buffer that alternates between the
// spatial domain and the "row spectrum" domain (FFT along x done).  One slice
// step is two passes:
//   row pass:    IFFT_x -> u_{i+1} = t_i * v (optionally recorded) -> FFT_x
//   column pass: FFT_y -> x H(dz) -> IFFT_y -> 1/(py px)    (prop2d column kernel)
// so the thin-sample product of slice i and both row transforms share one
// read and one write of the field.  The adjoint runs the same loop backwards:
//   row pass:    IFFT_x -> g_{i+1}; dL/d dn_i = k dz Im(g conj u_{i+1}),
//                dL/d abs_i = -k dz Re(g conj u_{i+1}); g *= conj(t_i) -> FFT_x
//   column pass: FFT_y -> x conj(H) = H(-dz) -> IFFT_y
// with g = dL/dRe(u) + i dL/dIm(u).  The forward fields u_{i+1} come from a
// recomputation of each checkpoint segment.
#pragma once

#include "prop2d.cuh"

namespace cx {

// MS_FLUOR: the fluorescent forward step (samples.py:387-404), transmittance
// and source before the propagation: v <- v exp(i k dz dn_i) + fl_i exp(i ph_i)
enum MsMode { MS_LOAD = 0, MS_FWD = 1, MS_BWD = 2, MS_FINAL = 3, MS_FLUOR = 4 };

struct MsArgs {
  int ny, nx, pad_y, pad_x, py, px;
  int mode, precision, slice, record;
  double lam, dz;
  float kdz_f;          // 2 pi dz / lam rounded once to float
  int sy, sx, oy, ox;   // MS_LOAD source: (sy, sx) matrix placed at offset (oy, ox) of the padded grid
  const float* dn;      // (D, ny, nx) refractive-index change (unpadded)
  const float* ab;      // (D, ny, nx) absorption (unpadded)
  const float2* src;    // MS_LOAD source
  float2* buf;          // (py, px) state
  float2* rec;          // record target (py, px), spatial domain
  const float2* rec_u;  // MS_BWD: u_{i+1} (py, px), spatial domain
  float* gdn;           // MS_BWD: dL/d dn_i  (ny, nx)
  float* gab;           // MS_BWD: dL/d abs_i (ny, nx)
  float2* dst;          // MS_FINAL: (ny, nx) crop of the padded grid
  const float2* twg;  // device twiddle tables (ensure_twiddles)
  const float* fl;      // MS_FLUOR: (D, ny, nx) fluorescence amplitude
  const float* ph;      // MS_FLUOR: (D, ny, nx) random phases
  float load_scale;     // MS_LOAD: factor on the source (1 / px when a row pass follows the load)
};

// thin-sample transmittance t = exp(i 2 pi dz / lam (dn + i abs))
__device__ __forceinline__ float2 ms_transmittance(const MsArgs& a, float dn, float ab) {
  if (a.precision == CX_PREC_REF32) {
    // 1j * 2 * pi (folded) * (dn + 1j abs) * thickness / lam, complex64 ops in order
    const float TWO_PI = 6.28318530717958647692f;
    const float th = (float)a.dz, lam = (float)a.lam;
    const float re = fd(fm(-fm(TWO_PI, ab), th), lam);
    const float im = fd(fm(fm(TWO_PI, dn), th), lam);
    float s, c;
    sincosf(im, &s, &c);
    const float m = expf(re);
    return make_float2(m * c, m * s);
  }
  // k dz is formed in FP64 (kdz_f); the slice phase k dz dn is a few tenths of
  // a radian for physical dn, so FP32 with the accurate sincosf suffices
  const float m = __expf(-a.kdz_f * ab);
  float s, c;
  sincosf(a.kdz_f * dn, &s, &c);
  return make_float2(m * c, m * s);
}

// shared memory of the row pass: the base row configuration plus, per team,
// a prefetch area for the slice's dn and abs rows (and, in the adjoint, the
// recorded forward field row)
template <int NX, int MODE>
struct MsRowCfg {
  using C = RowCfg<NX>;
  static constexpr int NXA = (NX + 3) & ~3;  // one row of floats, rounded to 16 bytes
  static constexpr int PF = (MODE == MS_FWD || MODE == MS_BWD || MODE == MS_FLUOR)
                                ? 2 * NXA + (MODE == MS_BWD ? 2 * NXA : 0) + (MODE == MS_FLUOR ? NXA : 0)
                                : 0;
  // bulk copies need 16-byte aligned shared destinations: the prefetch area
  // starts at the next 16-byte boundary after the transform buffers, and PF
  // (a multiple of 4 floats) keeps every team's area aligned; one mbarrier
  // per team follows
  static constexpr size_t PF_OFF = ((sizeof(float2) * ((size_t)C::TW + (size_t)C::TEAMS * Plan<NX>::LEN)) + 15) & ~(size_t)15;
  static_assert(PF % 4 == 0, "prefetch rows must keep 16-byte alignment");
  static constexpr size_t BAR_OFF = PF_OFF + sizeof(float) * (size_t)C::TEAMS * PF;
  static constexpr size_t SMEM = BAR_OFF + sizeof(uint64_t) * (size_t)C::TEAMS;
  static constexpr int POLLS = 1 << 20;
};

// Start copying dn / abs row yd of the slice (and the recorded field row) into
// the team's prefetch area: one lane arms the team's mbarrier with the byte
// count and issues one bulk (TMA) copy per row; returns false when the rows
// are not 16-byte aligned (the caller then reads them from global memory)
template <int NX, int MODE>
__device__ __forceinline__ bool ms_prefetch(const MsArgs& a, float* pf, uint64_t* bar, int yd, int y, int lane) {
  const size_t off = (size_t)a.slice * a.ny * a.nx + (size_t)yd * a.nx;
  const float* dn = a.dn + off;
  // MS_FLUOR: the second and third rows are the fluorescence and the phases
  const float* ab = (MODE == MS_FLUOR ? a.fl : a.ab) + off;
  bool ok = (a.nx % 4 == 0) && ((reinterpret_cast<size_t>(dn) & 15) == 0) && ((reinterpret_cast<size_t>(ab) & 15) == 0);
  const float* ph = MODE == MS_FLUOR ? a.ph + off : nullptr;
  if constexpr (MODE == MS_FLUOR) ok = ok && ((reinterpret_cast<size_t>(ph) & 15) == 0);
  const float2* u = nullptr;
  if constexpr (MODE == MS_BWD) {
    u = a.rec_u + (size_t)y * a.px;
    ok = ok && (a.px % 2 == 0) && ((reinterpret_cast<size_t>(u) & 15) == 0);
  }
  if (!ok) return false;
  constexpr int NXA = MsRowCfg<NX, MODE>::NXA;
  if (lane == 0) {
    const unsigned rb = (unsigned)a.nx * 4u;
    unsigned bytes = 2u * rb;
    if constexpr (MODE == MS_FLUOR) bytes += rb;
    if constexpr (MODE == MS_BWD) bytes += (unsigned)a.px * 8u;
    bulk_fence();  // the previous row's reads of this area precede the new writes
    bulk_expect(bar, bytes);
    // read once per pass: evict first (the field state and the propagator stay in L2)
    const uint64_t pol = l2_evict_first();
    bulk_copy_g2s_hint(pf, dn, rb, bar, pol);
    bulk_copy_g2s_hint(pf + NXA, ab, rb, bar, pol);
    if constexpr (MODE == MS_FLUOR) bulk_copy_g2s_hint(pf + 2 * NXA, ph, rb, bar, pol);
    if constexpr (MODE == MS_BWD) bulk_copy_g2s_hint(pf + 2 * NXA, u, (unsigned)a.px * 8u, bar, pol);
  }
  return true;
}

template <int NX, int MODE>
__global__ void __launch_bounds__(RowCfg<NX>::THREADS, RowCfg<NX>::MINB) k_ms_rows(MsArgs a) {
  using C = RowCfg<NX>;
  extern __shared__ __align__(16) float2 sm[];
  float2* tw = sm;
  load_twiddles<NX>(tw, a.twg, threadIdx.x, blockDim.x);
  __syncthreads();
  const int team = threadIdx.x / C::LPV, lane = threadIdx.x % C::LPV;
  float2* s = sm + C::TW + team * Plan<NX>::LEN;
  float* pf = reinterpret_cast<float*>(reinterpret_cast<char*>(sm) + MsRowCfg<NX, MODE>::PF_OFF) +
              (size_t)team * MsRowCfg<NX, MODE>::PF;
  uint64_t* bar = reinterpret_cast<uint64_t*>(reinterpret_cast<char*>(sm) + MsRowCfg<NX, MODE>::BAR_OFF) + team;
  if constexpr (MODE == MS_FWD || MODE == MS_BWD || MODE == MS_FLUOR) {
    if (lane == 0) bulk_mbar_init(bar);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    __syncthreads();
  }
  unsigned bphase = 0;  // parity of this team's next prefetch completion
  // MS_FINAL only produces the cropped rows
  const int r0 = MODE == MS_FINAL ? a.pad_y : 0;
  const int nrows = MODE == MS_FINAL ? a.ny : a.py;
  const long total = nrows;
  const size_t plane_d = (size_t)a.slice * a.ny * a.nx;
  const double kdz = 6.283185307179586476925286766559 * a.dz / a.lam;
  for (long base = (long)blockIdx.x * C::TEAMS; base < total; base += (long)gridDim.x * C::TEAMS) {
    const long item = base + team;
    if (item >= total) continue;
    const int y = r0 + (int)item;
    const int yd = y - a.pad_y;
    const bool yin = yd >= 0 && yd < a.ny;
    float2* row = a.buf + (size_t)y * a.px;
    if constexpr (MODE == MS_LOAD) {
      const int ys = y - a.oy;
      const bool rin = ys >= 0 && ys < a.sy;
      const float2* srow = a.src + (size_t)(rin ? ys : 0) * a.sx;
      float2* rrow = a.rec ? a.rec + (size_t)y * a.px : nullptr;
      auto load = [&](int n) -> float2 {
        const int xs = n - a.ox;
        const float2 v = (rin && xs >= 0 && xs < a.sx) ? cscale(srow[xs], a.load_scale) : make_float2(0.f, 0.f);
        if (a.record) rrow[n] = v;
        return v;
      };
      auto store = [&](int k, float2 v, int) { row[k] = v; };
      team_fft<NX, false>(s, tw, lane, team, load, store);
      continue;
    }
    // inverse FFT along x of the row spectrum
    auto load_row = [&](int n) -> float2 { return row[n]; };
    if constexpr (MODE == MS_FINAL) {
      float2* drow = a.dst + (size_t)yd * a.nx;
      auto store = [&](int k, float2 v, int) {
        const int xd = k - a.pad_x;
        if (xd >= 0 && xd < a.nx) drow[xd] = v;
      };
      team_fft<NX, true>(s, tw, lane, team, load_row, store);
      continue;
    }
    if constexpr (MODE == MS_FWD || MODE == MS_BWD || MODE == MS_FLUOR) {
    // the slice's rows stream into shared memory while the inverse transform runs
    bool pre = yin && ms_prefetch<NX, MODE>(a, pf, bar, yd, y, lane);
    auto sst = [&](int k, float2 v, int) { s[pad_idx(k)] = v; };
    team_fft<NX, true>(s, tw, lane, team, load_row, sst);
    if (pre) {
      // the rows landed during the inverse transform; past the (generous)
      // poll limit the lane reads them from global memory instead
      pre = bulk_wait(bar, bphase, MsRowCfg<NX, MODE>::POLLS);
      bphase ^= 1u;
    }
    team_sync<C::LPV>(team);
    if constexpr (MODE == MS_FLUOR) {
      constexpr int NXA = MsRowCfg<NX, MODE>::NXA;
#pragma unroll 2
      for (int k = lane; k < NX; k += C::LPV) {
        float2 v = s[pad_idx(k)];
        const int xd = k - a.pad_x;
        if (yin && xd >= 0 && xd < a.nx) {
          const size_t idx = plane_d + (size_t)yd * a.nx + xd;
          const float dnv = pre ? pf[xd] : a.dn[idx];
          const float flv = pre ? pf[NXA + xd] : a.fl[idx];
          const float phv = pre ? pf[2 * NXA + xd] : a.ph[idx];
          float sp, cp;
          sincosf(phv, &sp, &cp);
          v = cmul(v, ms_transmittance(a, dnv, 0.f));
          v = make_float2(v.x + flv * cp, v.y + flv * sp);
        }
        s[pad_idx(k)] = v;
      }
    } else if constexpr (MODE == MS_FWD) {
      float2* rrow = a.record ? a.rec + (size_t)y * a.px : nullptr;
      const uint64_t rpol = l2_evict_first();  // records are read back once, by the adjoint
#pragma unroll 2
      for (int k = lane; k < NX; k += C::LPV) {
        float2 v = s[pad_idx(k)];
        const int xd = k - a.pad_x;
        if (yin && xd >= 0 && xd < a.nx) {
          const size_t idx = plane_d + (size_t)yd * a.nx + xd;
          const float dnv = pre ? pf[xd] : a.dn[idx];
          const float abv = pre ? pf[MsRowCfg<NX, MODE>::NXA + xd] : a.ab[idx];
          v = cmul(v, ms_transmittance(a, dnv, abv));
        }
        if (a.record) st_hint(rrow + k, v, rpol);
        s[pad_idx(k)] = v;
      }
    } else {  // MS_BWD
      const float2* urow = a.rec_u + (size_t)y * a.px;
      const float2* purow = reinterpret_cast<const float2*>(pf + 2 * MsRowCfg<NX, MODE>::NXA);
#pragma unroll 2
      for (int k = lane; k < NX; k += C::LPV) {
        float2 g = s[pad_idx(k)];
        const int xd = k - a.pad_x;
        if (yin && xd >= 0 && xd < a.nx) {
          const size_t idx = plane_d + (size_t)yd * a.nx + xd;
          const float2 u = pre ? purow[k] : urow[k];
          // w = g * conj(u)
          const float wr = g.x * u.x + g.y * u.y, wi = g.y * u.x - g.x * u.y;
          const size_t gi = (size_t)yd * a.nx + xd;
          a.gdn[gi] = (float)(kdz * (double)wi);
          a.gab[gi] = (float)(-kdz * (double)wr);
          const float dnv = pre ? pf[xd] : a.dn[idx];
          const float abv = pre ? pf[MsRowCfg<NX, MODE>::NXA + xd] : a.ab[idx];
          g = cmul(g, cconj(ms_transmittance(a, dnv, abv)));
        }
        s[pad_idx(k)] = g;
      }
    }
    team_sync<C::LPV>(team);
    auto load2 = [&](int n) -> float2 { return s[pad_idx(n)]; };
    auto store2 = [&](int k, float2 v, int) { row[k] = v; };
    team_fft<NX, false>(s, tw, lane, team, load2, store2);
    }
  }
}

cx_status ms_dispatch_rows(int n, const MsArgs& a, cudaStream_t st);
// CX_PREC_SPLIT16 row passes on the tensor cores (multislice_tc.cu) where the
// padded row length is compiled in; other lengths and the fluorescent step
// keep the FP32 butterflies
bool ms_tc_rows_supported(int px, int mode);
cx_status ms_dispatch_rows_tc(const MsArgs& a, cudaStream_t st);
inline cx_status ms_rows(const MsArgs& a, cudaStream_t st) {
  return a.precision == CX_PREC_SPLIT16 && ms_tc_rows_supported(a.px, a.mode) ? ms_dispatch_rows_tc(a, st)
                                                                              : ms_dispatch_rows(a.px, a, st);
}

}  // namespace cx
