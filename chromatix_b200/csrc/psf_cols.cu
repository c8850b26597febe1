// Column pass of the fused PSF (see psf.cuh).
#include "psf.cuh"

namespace cx {

template <int NY>
static cx_status launch_psf_cols(const PsfArgs& a, cudaStream_t st) {
  using C = ColCfg<NY>;
  const int q = psf_edge_q(a, true, NY, Plan<NY>::P.r[0]);
  auto k = q == 3 ? k_psf_cols<NY, 3> : q == 4 ? k_psf_cols<NY, 4> : q == 6 ? k_psf_cols<NY, 6> : k_psf_cols<NY, 0>;
  CX_CUDA_TRY(set_smem(k, PsfColCfg<NY>::SMEM));
  const long items = (long)((a.nx + C::V - 1) / C::V) * a.zc;
  const int grid = persistent_grid(k, C::THREADS, PsfColCfg<NY>::SMEM, items);
  k<<<grid, C::THREADS, PsfColCfg<NY>::SMEM, st>>>(a);
  CX_LAUNCH_CHECK();
  return CX_OK;
}

cx_status psf_dispatch_cols(int n, const PsfArgs& a, cudaStream_t st) {
  switch (n) {
#define CX_CASE_(N) \
  case N:           \
    return launch_psf_cols<N>(a, st);
    CX_FOR_EACH_SIZE(CX_CASE_)
#undef CX_CASE_
  }
  set_error("FFT length %d is not supported", n);
  return CX_ERR_UNSUPPORTED;
}

}  // namespace cx
