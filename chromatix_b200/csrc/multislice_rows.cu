// Row passes of the multislice loop (see multislice.cuh).
#include "multislice.cuh"

namespace cx {

template <int NX, int MODE>
static cx_status launch_ms_rows_mode(const MsArgs& a, cudaStream_t st) {
  using C = RowCfg<NX>;
  constexpr size_t SMEM = MsRowCfg<NX, MODE>::SMEM;
  auto k = k_ms_rows<NX, MODE>;
  CX_CUDA_TRY(set_smem(k, SMEM));
  const long rows = a.mode == MS_FINAL ? a.ny : a.py;
  const long items = (rows + C::TEAMS - 1) / C::TEAMS;
  k<<<persistent_grid(k, C::THREADS, SMEM, items), C::THREADS, SMEM, st>>>(a);
  CX_LAUNCH_CHECK();
  return CX_OK;
}

template <int NX>
static cx_status launch_ms_rows(const MsArgs& a, cudaStream_t st) {
  switch (a.mode) {
    case MS_LOAD:
      return launch_ms_rows_mode<NX, MS_LOAD>(a, st);
    case MS_FWD:
      return launch_ms_rows_mode<NX, MS_FWD>(a, st);
    case MS_BWD:
      return launch_ms_rows_mode<NX, MS_BWD>(a, st);
    case MS_FLUOR:
      return launch_ms_rows_mode<NX, MS_FLUOR>(a, st);
    default:
      return launch_ms_rows_mode<NX, MS_FINAL>(a, st);
  }
}

cx_status ms_dispatch_rows(int n, const MsArgs& a, cudaStream_t st) {
  switch (n) {
#define CX_CASE_(N) \
  case N:           \
    return launch_ms_rows<N>(a, st);
    CX_FOR_EACH_SIZE(CX_CASE_)
#undef CX_CASE_
  }
  set_error("FFT length %d is not supported", n);
  return CX_ERR_UNSUPPORTED;
}

}  // namespace cx
