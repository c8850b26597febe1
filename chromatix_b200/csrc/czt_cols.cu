// Chirp-Z transform along a strided axis, column tiles (see czt.cuh).
#include "czt.cuh"

namespace cx {

template <int L>
static cx_status launch_czt_cols(const CztArgs& a, cudaStream_t st) {
  using C = ColCfg<L>;
  auto k = k_czt_cols<L>;
  const long items = (long)((a.inner + C::V - 1) / C::V) * (a.n_vec / a.inner);
  k<<<persistent_grid(k, C::THREADS, C::SMEM, items), C::THREADS, C::SMEM, st>>>(a);
  CX_LAUNCH_CHECK();
  return CX_OK;
}

cx_status czt_dispatch_cols(int L, const CztArgs& a, cudaStream_t st) {
  switch (L) {
#define CX_CASE_(N) \
  case N:           \
    return launch_czt_cols<N>(a, st);
    CX_FOR_EACH_1D_SIZE(CX_CASE_)
#undef CX_CASE_
  }
  set_error("FFT length %d is not supported", L);
  return CX_ERR_UNSUPPORTED;
}

}  // namespace cx
