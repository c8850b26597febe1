// Column pass of the chirped optical FFT (see optfft.cuh).
#include "optfft.cuh"

namespace cx {

template <int NY>
__global__ void __launch_bounds__(ColCfg<NY>::THREADS, ColCfg<NY>::MINB) k_opt_cols(const float2* __restrict__ T,
                                                                 float2* __restrict__ out, OptArgs a) {
  using C = ColCfg<NY>;
  constexpr int V = C::V, LEN = C::LEN;
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* tile = sm + C::TW;
  load_twiddles<NY>(tw, a.twg, threadIdx.x, blockDim.x);
  const int team = threadIdx.x / C::LPV, lane = threadIdx.x % C::LPV;
  float2* s = tile + team * LEN;
  const int tiles_x = (a.px + V - 1) / V;
  const long total = (long)tiles_x * a.n_out_planes;
  for (long t = blockIdx.x; t < total; t += gridDim.x) {
    const int q = (int)(t / tiles_x);
    const int x0 = (int)(t % tiles_x) * V;
    const cx_fft_plane pl = a.planes[q];
    __syncthreads();
    for (int idx = threadIdx.x; idx < a.py * V; idx += blockDim.x) {
      const int yy = idx / V, c = idx % V, x = x0 + c;
      tile[c * LEN + pad_idx(yy)] = x < a.px ? T[((size_t)q * a.py + yy) * a.px + x] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    const int kx = x0 + team;
    const int col = add_mod(kx, a.px / 2, a.px);  // fftshift along x
    const double rx = pl.dx_out * ((double)col - 0.5 * a.px) + pl.ox;
    const float2 post = make_float2((float)pl.post_re, (float)pl.post_im);
    auto load = [&](int n) -> float2 { return s[pad_idx(n)]; };
    // the tile stays in FFT order (the staged store updates it in place);
    // the fftshift along y is applied by the final copy
    const float2* hcol = a.H ? a.H + (size_t)q * a.py * a.px + kx : nullptr;
    auto store = [&](int k, float2 v, int) {
      const int row = add_mod(k, a.py / 2, a.py);  // output row of bin k (fftshift along y)
      if (hcol && kx < a.px) v = cmul(v, hcol[(size_t)k * a.px]);
      if (pl.conj) v = cconj(v);
      v = cmul(post, v);
      if (pl.chirp_out != 0.0 || pl.pupil_out_r2 > 0.0) {
        const double ry = pl.dy_out * ((double)row - 0.5 * a.py) + pl.oy;
        if (pl.chirp_out != 0.0) v = cmul(v, chirp(pl.chirp_out, ry, rx));
        // output-grid pupil (the adjoint of the input pupil of ff_lens)
        if (pl.pupil_out_r2 > 0.0 && ry * ry + rx * rx > pl.pupil_out_r2) v = make_float2(0.f, 0.f);
      }
      s[pad_idx(k)] = v;
    };
    team_fft_ex<NY, false, false, true, C::LPV, C::CTA>(s, tw, lane, team, load, store);
    __syncthreads();
    const int b = q / a.W, w = q % a.W;
    for (int idx = threadIdx.x; idx < a.oy_n * V; idx += blockDim.x) {
      const int r = idx / V, c = idx % V, x = x0 + c;
      if (x >= a.px) continue;
      const int colo = add_mod(x, a.px / 2, a.px) - a.crop_x;
      if (colo < 0 || colo >= a.ox_n) continue;
      const int k = add_mod(r + a.crop_y, a.py - a.py / 2, a.py);  // FFT bin of output row r
      out[(((size_t)b * a.oy_n + r) * a.ox_n + colo) * a.W + w] = tile[c * LEN + pad_idx(k)];
    }
  }
}

template <int NY>
static cx_status launch_opt_cols(const float2* T, float2* out, const OptArgs& a, cudaStream_t st) {
  using C = ColCfg<NY>;
  auto k = k_opt_cols<NY>;
  CX_CUDA_TRY(set_smem(k, C::SMEM));
  const long items = (long)((a.px + C::V - 1) / C::V) * a.n_out_planes;
  k<<<persistent_grid(k, C::THREADS, C::SMEM, items), C::THREADS, C::SMEM, st>>>(T, out, a);
  CX_LAUNCH_CHECK();
  return CX_OK;
}

cx_status opt_dispatch_cols(int n, const float2* T, float2* out, const OptArgs& a, cudaStream_t st) {
  switch (n) {
#define CX_CASE_(N) \
  case N:           \
    return launch_opt_cols<N>(T, out, a, st);
    CX_FOR_EACH_SIZE(CX_CASE_)
#undef CX_CASE_
  }
  set_error("FFT length %d is not supported", n);
  return CX_ERR_UNSUPPORTED;
}
}  // namespace cx
