// Row-direction kernels of the plane-wise Fourier convolution (conv.cuh):
// the forward r2c rows and the final c2r rows, one instance per half row
// length M.
#include "conv.cuh"

namespace cx {

template <int M>
static cx_status launch_rows(const ConvArgs& a, cudaStream_t st) {
  using C = RowCfg<M>;
  auto k = k_conv_rows<M>;
  CX_CUDA_TRY(set_smem(k, C::SMEM));
  const long items = ((long)a.zc * (a.h + a.kh) + C::TEAMS - 1) / C::TEAMS;
  k<<<persistent_grid(k, C::THREADS, C::SMEM, items), C::THREADS, C::SMEM, st>>>(a);
  CX_LAUNCH_CHECK();
  return CX_OK;
}

template <int M>
static cx_status launch_fin_rows(const ConvArgs& a, cudaStream_t st) {
  using Q = ConvFinCfg<M>;
  auto k = k_conv_fin_rows<M>;
  CX_CUDA_TRY(set_smem(k, Q::SMEM));
  const long items = (a.h + Q::V - 1) / Q::V;
  k<<<persistent_grid(k, Q::THREADS, Q::SMEM, items), Q::THREADS, Q::SMEM, st>>>(a);
  CX_LAUNCH_CHECK();
  return CX_OK;
}

cx_status conv_dispatch_rows(int m, const ConvArgs& a, cudaStream_t st) {
  switch (m) {
#define CX_CONV_CASE_(N) \
  case N:                \
    return launch_rows<N>(a, st);
    CX_CONV_M_SIZES(CX_CONV_CASE_)
#undef CX_CONV_CASE_
  }
  set_error("convolution half row length %d is not supported", m);
  return CX_ERR_UNSUPPORTED;
}

cx_status conv_dispatch_fin_rows(int m, const ConvArgs& a, cudaStream_t st) {
  switch (m) {
#define CX_CONV_CASE_(N) \
  case N:                \
    return launch_fin_rows<N>(a, st);
    CX_CONV_M_SIZES(CX_CONV_CASE_)
#undef CX_CONV_CASE_
  }
  set_error("convolution half row length %d is not supported", m);
  return CX_ERR_UNSUPPORTED;
}

}  // namespace cx
