// Column-direction kernels of the plane-wise Fourier convolution (conv.cuh):
// the forward column transforms with the plane-summed product and the final
// column inverse, one instance per column length P.
#include "conv.cuh"

namespace cx {

template <int P>
static cx_status launch_cols(const ConvArgs& a, cudaStream_t st) {
  using Q = ConvColCfg<P>;
  auto k = k_conv_cols<P>;
  CX_CUDA_TRY(set_smem(k, Q::SMEM));
  const long items = (a.NC + Q::V - 1) / Q::V;
  k<<<persistent_grid(k, Q::THREADS, Q::SMEM, items), Q::THREADS, Q::SMEM, st>>>(a);
  CX_LAUNCH_CHECK();
  return CX_OK;
}

template <int P>
static cx_status launch_fin_cols(const ConvArgs& a, cudaStream_t st) {
  using C = RowCfg<P>;
  auto k = k_conv_fin_cols<P>;
  CX_CUDA_TRY(set_smem(k, C::SMEM));
  const long items = ((long)a.NC + C::TEAMS - 1) / C::TEAMS;
  k<<<persistent_grid(k, C::THREADS, C::SMEM, items), C::THREADS, C::SMEM, st>>>(a);
  CX_LAUNCH_CHECK();
  return CX_OK;
}

cx_status conv_dispatch_cols(int p, const ConvArgs& a, cudaStream_t st) {
  switch (p) {
#define CX_CONV_CASE_(N) \
  case N:                \
    return launch_cols<N>(a, st);
    CX_CONV_P_SIZES(CX_CONV_CASE_)
#undef CX_CONV_CASE_
  }
  set_error("convolution column length %d is not supported", p);
  return CX_ERR_UNSUPPORTED;
}

int conv_col_tile(int p) {
  switch (p) {
#define CX_CONV_CASE_(N) \
  case N:                \
    return ConvColCfg<N>::V;
    CX_CONV_P_SIZES(CX_CONV_CASE_)
#undef CX_CONV_CASE_
  }
  return 0;
}

cx_status conv_dispatch_fin_cols(int p, const ConvArgs& a, cudaStream_t st) {
  switch (p) {
#define CX_CONV_CASE_(N) \
  case N:                \
    return launch_fin_cols<N>(a, st);
    CX_CONV_P_SIZES(CX_CONV_CASE_)
#undef CX_CONV_CASE_
  }
  set_error("convolution column length %d is not supported", p);
  return CX_ERR_UNSUPPORTED;
}

}  // namespace cx
