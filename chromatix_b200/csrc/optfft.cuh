// Centred optical FFT with fused chirps, pupil, padding and crop.
//
// Reference: functional/convenience.py:9-59 (optical_fft), utils/fft.py:8-20
// (fftshift(fft2(ifftshift(x)))), functional/lenses.py:64-95 / 159-198
// (ff_lens, df_lens), functional/propagation.py:34-82 (transform_propagate).
//
// pass A  rows: zero pad, input chirp, pupil, conjugation, complex pre-factor
//         evaluated in the loader; ifftshift is an index remap; row FFT.
// pass B  V-column tiles: column FFT; fftshift, conjugation, post factor,
//         output chirp and crop in the store.
#pragma once
#include "host.cuh"

namespace cx {

struct OptArgs {
  int ny, nx, pad_y, pad_x, py, px, crop_y, crop_x, oy_n, ox_n, W;
  int n_in_planes, n_out_planes, precision;
  const cx_fft_plane* planes;
  const float2* H;  // optional propagator table (planar, FFT order), multiplied before the fftshift
  const float2* twg;  // device twiddle tables (ensure_twiddles)
};

__device__ __forceinline__ float2 chirp(double c, double ry, double rx) {
  return expi_reduced(c * (ry * ry + rx * rx));
}

cx_status opt_dispatch_rows(int n, const float2* u, float2* T, const OptArgs& a, cudaStream_t st);
cx_status opt_dispatch_cols(int n, const float2* T, float2* out, const OptArgs& a, cudaStream_t st);
}  // namespace cx
