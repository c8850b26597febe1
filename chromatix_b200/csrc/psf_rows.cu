// Row pass of the fused PSF (see psf.cuh).
#include "psf.cuh"

namespace cx {

template <int NX>
static cx_status launch_psf_rows(const PsfArgs& a, cudaStream_t st) {
  const long rows = (long)a.zc * a.rowsum;
  if (a.precision != CX_PREC_REF32) {
    using C = PsfRowCfg<NX>;
    const int q = psf_edge_q(a, false, NX, Plan<NX>::P.r[0]);
    auto k = q == 3   ? k_psf_rows_tab<NX, 3>
             : q == 4 ? k_psf_rows_tab<NX, 4>
             : q == 6 ? k_psf_rows_tab<NX, 6>
                      : k_psf_rows_tab<NX, 0>;
    CX_CUDA_TRY(set_smem(k, C::SMEM));
    const int grid = persistent_grid(k, C::THREADS, C::SMEM, (rows + C::TEAMS - 1) / C::TEAMS);
    k<<<grid, C::THREADS, C::SMEM, st>>>(a);
  } else {
    using C = RowCfg<NX>;
    auto k = k_psf_rows<NX>;
    CX_CUDA_TRY(set_smem(k, C::SMEM));
    const int grid = persistent_grid(k, C::THREADS, C::SMEM, (rows + C::TEAMS - 1) / C::TEAMS);
    k<<<grid, C::THREADS, C::SMEM, st>>>(a);
  }
  CX_LAUNCH_CHECK();
  return CX_OK;
}

cx_status psf_dispatch_rows(int n, const PsfArgs& a, cudaStream_t st) {
  switch (n) {
#define CX_CASE_(N) \
  case N:           \
    return launch_psf_rows<N>(a, st);
    CX_FOR_EACH_SIZE(CX_CASE_)
#undef CX_CASE_
  }
  set_error("FFT length %d is not supported", n);
  return CX_ERR_UNSUPPORTED;
}

}  // namespace cx
