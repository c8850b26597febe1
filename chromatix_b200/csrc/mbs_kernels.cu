// Launchers of the modified-Born-series passes (kernels in mbs.cuh).
#include "mbs.cuh"

namespace cx {

// 3D grid lengths compiled for the MBS passes
#define CX_MBS_SIZES(X) \
  X(16) X(20) X(24) X(28) X(32) X(40) X(48) X(56) X(64) X(80) X(96) X(112) X(128) X(160) X(192) X(224) X(256) \
  X(320) X(384) X(448) X(512)

template <int N, int MODE>
static cx_status launch_z(const MbsArgs& a, cudaStream_t st) {
  using C = RowCfg<N>;
  constexpr size_t SMEM = MbsZCfg<N, MODE>::SMEM;
  auto k = k_mbs_z<N, MODE>;
  CX_CUDA_TRY(set_smem(k, SMEM));
  const long items = ((long)a.X * a.Y + C::TEAMS - 1) / C::TEAMS;
  k<<<persistent_grid(k, C::THREADS, SMEM, items), C::THREADS, SMEM, st>>>(a);
  CX_LAUNCH_CHECK();
  return CX_OK;
}

template <int N>
static cx_status launch_z_any(int mode, const MbsArgs& a, cudaStream_t st) {
  switch (mode) {
    case MBS_Z_DISC:
      return launch_z<N, MBS_Z_DISC>(a, st);
    case MBS_Z_SCALE:
      return launch_z<N, MBS_Z_SCALE>(a, st);
    case MBS_ZI_STEP:
      return launch_z<N, MBS_ZI_STEP>(a, st);
    default:
      return launch_z<N, MBS_ZI_PREC>(a, st);
  }
}

template <int N, bool INV>
static cx_status launch_cols(const MbsArgs& a, long n_outer, int inner, long ostride, long E, cudaStream_t st) {
  using C = MbsColCfg<N>;
  constexpr size_t SMEM = C::SMEM;
  auto k = k_mbs_cols<N, INV>;
  CX_CUDA_TRY(set_smem(k, SMEM));
  const long items = (long)((inner + C::V - 1) / C::V) * n_outer;
  k<<<persistent_grid(k, C::THREADS, SMEM, items), C::THREADS, SMEM, st>>>(a, n_outer, inner, ostride, E);
  CX_LAUNCH_CHECK();
  return CX_OK;
}

template <int N>
static cx_status launch_x(const MbsArgs& a, cudaStream_t st) {
  using Q = MbsXCfg<N>;
  auto k = k_mbs_x<N>;
  CX_CUDA_TRY(set_smem(k, Q::SMEM));
  const long items = ((long)a.Y * a.Z + Q::V - 1) / Q::V;
  k<<<persistent_grid(k, Q::THREADS, Q::SMEM, items), Q::THREADS, Q::SMEM, st>>>(a);
  CX_LAUNCH_CHECK();
  return CX_OK;
}

bool mbs_size_supported(int n) {
  switch (n) {
#define CX_CASE_(N) case N:
    CX_MBS_SIZES(CX_CASE_)
#undef CX_CASE_
    return true;
    default:
      return false;
  }
}

cx_status mbs_dispatch_z(int n, int mode, const MbsArgs& a, cudaStream_t st) {
  switch (n) {
#define CX_CASE_(N) \
  case N:           \
    return launch_z_any<N>(mode, a, st);
    CX_MBS_SIZES(CX_CASE_)
#undef CX_CASE_
  }
  set_error("MBS grid length %d is not supported", n);
  return CX_ERR_UNSUPPORTED;
}

cx_status mbs_dispatch_cols(int n, bool inv, const MbsArgs& a, long n_outer, int inner, long ostride, long E,
                            cudaStream_t st) {
  switch (n) {
#define CX_CASE_(N)                                                                       \
  case N:                                                                                 \
    return inv ? launch_cols<N, true>(a, n_outer, inner, ostride, E, st)                  \
               : launch_cols<N, false>(a, n_outer, inner, ostride, E, st);
    CX_MBS_SIZES(CX_CASE_)
#undef CX_CASE_
  }
  set_error("MBS grid length %d is not supported", n);
  return CX_ERR_UNSUPPORTED;
}

cx_status mbs_dispatch_x(int n, const MbsArgs& a, cudaStream_t st) {
  switch (n) {
#define CX_CASE_(N) \
  case N:           \
    return launch_x<N>(a, st);
    CX_MBS_SIZES(CX_CASE_)
#undef CX_CASE_
  }
  set_error("MBS grid length %d is not supported", n);
  return CX_ERR_UNSUPPORTED;
}

}  // namespace cx
