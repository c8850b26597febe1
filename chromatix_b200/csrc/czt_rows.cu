// Chirp-Z transform, one team per vector (see czt.cuh).
#include "czt.cuh"

namespace cx {

template <int L>
static cx_status launch_czt_rows(const CztArgs& a, cudaStream_t st) {
  using C = RowCfg<L>;
  auto k = k_czt_rows<L>;
  const long items = (a.n_vec + C::TEAMS - 1) / C::TEAMS;
  k<<<persistent_grid(k, C::THREADS, C::SMEM, items), C::THREADS, C::SMEM, st>>>(a);
  CX_LAUNCH_CHECK();
  return CX_OK;
}

cx_status czt_dispatch_rows(int L, const CztArgs& a, cudaStream_t st) {
  switch (L) {
#define CX_CASE_(N) \
  case N:           \
    return launch_czt_rows<N>(a, st);
    CX_FOR_EACH_1D_SIZE(CX_CASE_)
#undef CX_CASE_
  }
  set_error("FFT length %d is not supported", L);
  return CX_ERR_UNSUPPORTED;
}

}  // namespace cx
