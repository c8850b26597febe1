// Row passes of the Fourier-multiplier propagation (see prop2d.cuh).
#include "prop2d.cuh"

namespace cx {

template <int NX>
static cx_status launch_rows_fwd(const float2* u, float2* T, const Prop2DArgs& a, cudaStream_t st) {
  using C = RowCfg<NX>;
  auto k = k_prop_rows_fwd<NX, false>;
  if constexpr (band_compiled<NX>()) {
    if (in_center_band(NX, a.pad_x, a.nx)) k = k_prop_rows_fwd<NX, true>;
  }
  CX_CUDA_TRY(set_smem(k, C::SMEM));
  const long items = ((long)a.n_in_planes * a.ny + C::TEAMS - 1) / C::TEAMS;
  const int grid = persistent_grid(k, C::THREADS, C::SMEM, items);
  k<<<grid, C::THREADS, C::SMEM, st>>>(u, T, a);
  CX_LAUNCH_CHECK();
  return CX_OK;
}

template <int NX>
static cx_status launch_rows_inv(const float2* T2, float2* out, const Prop2DArgs& a, cudaStream_t st) {
  using C = RowCfg<NX>;
  auto k = k_prop_rows_inv<NX>;
  CX_CUDA_TRY(set_smem(k, C::SMEM));
  const long items = ((long)a.n_out_planes * a.out_ny + C::TEAMS - 1) / C::TEAMS;
  const int grid = persistent_grid(k, C::THREADS, C::SMEM, items);
  k<<<grid, C::THREADS, C::SMEM, st>>>(T2, out, a);
  CX_LAUNCH_CHECK();
  return CX_OK;
}

cx_status dispatch_rows_fwd(int n, const float2* u, float2* T, const Prop2DArgs& a, cudaStream_t st) {
  switch (n) {
#define CX_CASE_(N) \
  case N:           \
    return launch_rows_fwd<N>(u, T, a, st);
    CX_FOR_EACH_PROP_SIZE(CX_CASE_)
#undef CX_CASE_
  }
  set_error("FFT length %d is not supported", n);
  return CX_ERR_UNSUPPORTED;
}

cx_status dispatch_rows_inv(int n, const float2* T2, float2* out, const Prop2DArgs& a, cudaStream_t st) {
  switch (n) {
#define CX_CASE_(N) \
  case N:           \
    return launch_rows_inv<N>(T2, out, a, st);
    CX_FOR_EACH_PROP_SIZE(CX_CASE_)
#undef CX_CASE_
  }
  set_error("FFT length %d is not supported", n);
  return CX_ERR_UNSUPPORTED;
}

}  // namespace cx
