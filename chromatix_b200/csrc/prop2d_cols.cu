// Column pass of the Fourier-multiplier propagation (see prop2d.cuh).
#include "prop2d.cuh"

namespace cx {

template <int NY>
static cx_status launch_cols(const float2* T, float2* T2, const Prop2DArgs& a, cudaStream_t st) {
  using C = ColCfg<NY>;
  auto k = k_prop_cols<NY, false>;
  size_t smem = C::SMEM;
  const bool band = band_compiled<NY>() && in_center_band(NY, a.pad_y, a.ny);
  if constexpr (band_compiled<NY>()) {
    if (band) k = k_prop_cols<NY, true>;
  }
  if constexpr (PropColHt<NY>::FITS) {
    // a propagator table (prop_col mode 4) and no band pruning: stage H with the tile
    if (!band && a.kernel == CX_KERNEL_EXPLICIT && a.na_f2 < 0.0 && a.H) {
      k = k_prop_cols<NY, false, true>;
      smem = PropColHt<NY>::SMEM;
    }
  }
  CX_CUDA_TRY(set_smem(k, smem));
  const long items = (long)((a.px + C::V - 1) / C::V) * a.n_out_planes;
  const int grid = persistent_grid(k, C::THREADS, smem, items);
  k<<<grid, C::THREADS, smem, st>>>(T, T2, a);
  CX_LAUNCH_CHECK();
  return CX_OK;
}

cx_status dispatch_cols(int n, const float2* T, float2* T2, const Prop2DArgs& a, cudaStream_t st) {
  switch (n) {
#define CX_CASE_(N) \
  case N:           \
    return launch_cols<N>(T, T2, a, st);
    CX_FOR_EACH_PROP_SIZE(CX_CASE_)
#undef CX_CASE_
  }
  set_error("FFT length %d is not supported", n);
  return CX_ERR_UNSUPPORTED;
}

}  // namespace cx
