// Row pass of the chirped optical FFT (see optfft.cuh).
#include "optfft.cuh"

namespace cx {

template <int NX>
__global__ void __launch_bounds__(RowCfg<NX>::THREADS, RowCfg<NX>::MINB) k_opt_rows(const float2* __restrict__ u,
                                                                 float2* __restrict__ T, OptArgs a) {
  using C = RowCfg<NX>;
  extern __shared__ float2 sm[];
  float2* tw = sm;
  load_twiddles<NX>(tw, a.twg, threadIdx.x, blockDim.x);
  __syncthreads();
  const int team = threadIdx.x / C::LPV, lane = threadIdx.x % C::LPV;
  float2* s = sm + C::TW + team * Plan<NX>::LEN;
  const long total = (long)a.n_out_planes * a.py;
  for (long base = (long)blockIdx.x * C::TEAMS; base < total; base += (long)gridDim.x * C::TEAMS) {
    const long item = base + team;
    const bool valid = item < total;
    const int q = valid ? (int)(item / a.py) : 0;
    const int yy = valid ? (int)(item % a.py) : 0;
    const cx_fft_plane pl = a.planes[q];
    const int yp = add_mod(yy, a.py / 2, a.py);  // ifftshift: padded-grid row feeding FFT row yy
    const int y = yp - a.pad_y;
    const bool row_data = valid && y >= 0 && y < a.ny;
    const int b = pl.in_plane / a.W, w = pl.in_plane % a.W;
    const float2* src = u + ((size_t)b * a.ny + (row_data ? y : 0)) * a.nx * a.W + w;
    const double ry = pl.dy_in * ((double)yp - 0.5 * a.py) + pl.oy;
    const float2 pre = make_float2((float)pl.pre_re, (float)pl.pre_im);
    auto load = [&](int n) -> float2 {
      const int xp = add_mod(n, a.px / 2, a.px);
      const int x = xp - a.pad_x;
      if (!row_data || x < 0 || x >= a.nx) return make_float2(0.f, 0.f);
      float2 v = src[(size_t)x * a.W];
      const double rx = pl.dx_in * ((double)xp - 0.5 * a.px) + pl.ox;
      // circular_pupil tests |field.grid|^2, the grid including the origin (pupils.py:17-23)
      if (pl.pupil_r2 >= 0.0 && ry * ry + rx * rx > pl.pupil_r2) return make_float2(0.f, 0.f);
      if (pl.chirp_in != 0.0) v = cmul(v, chirp(pl.chirp_in, ry, rx));
      if (pl.conj) v = cconj(v);
      return cmul(pre, v);
    };
    float2* dst = T + ((size_t)q * a.py + yy) * a.px;
    auto store = [&](int k, float2 v, int) {
      if (valid) dst[k] = v;
    };
    team_fft_ex<NX, false, true, false>(s, tw, lane, team, load, store);
  }
}

template <int NX>
static cx_status launch_opt_rows(const float2* u, float2* T, const OptArgs& a, cudaStream_t st) {
  using C = RowCfg<NX>;
  auto k = k_opt_rows<NX>;
  CX_CUDA_TRY(set_smem(k, C::SMEM));
  const long items = ((long)a.n_out_planes * a.py + C::TEAMS - 1) / C::TEAMS;
  k<<<persistent_grid(k, C::THREADS, C::SMEM, items), C::THREADS, C::SMEM, st>>>(u, T, a);
  CX_LAUNCH_CHECK();
  return CX_OK;
}

cx_status opt_dispatch_rows(int n, const float2* u, float2* T, const OptArgs& a, cudaStream_t st) {
  switch (n) {
#define CX_CASE_(N) \
  case N:           \
    return launch_opt_rows<N>(u, T, a, st);
    CX_FOR_EACH_SIZE(CX_CASE_)
#undef CX_CASE_
  }
  set_error("FFT length %d is not supported", n);
  return CX_ERR_UNSUPPORTED;
}
}  // namespace cx
