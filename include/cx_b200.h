/*
 * cx_b200.h -- C ABI of the B200-native Chromatix propagation kernels.
 *
 * The reference (chromatix 0.5.0) is pure Python/JAX and has no native
 * interface; these entry points are what a jax.ffi / XLA FFI custom call for
 * each hot-path function binds.  Each declaration names the reference
 * function it replaces (paths relative to the chromatix repository root).
 *
 * Conventions
 *  - All field buffers are complex64 (interleaved float re, im), device
 *    memory owned by the caller, laid out like the reference's Field.u:
 *    (batch..., y, x) for a monochromatic field, (batch..., y, x, wv) for a
 *    chromatic one (wv innermost, stride n_wv).
 *  - Per-plane parameters (z, wavelength, spacing, ...) are an array of
 *    cx_plane in DEVICE memory, one entry per output (batch, wavelength)
 *    plane, so the same launch can be replayed from a CUDA graph with new
 *    values.
 *  - Scratch space is a caller-provided workspace of the size reported by
 *    the matching *_workspace_size call.  No entry point allocates device
 *    memory, synchronises the stream, or traps: errors come back as a
 *    cx_status and a thread-local message (cx_last_error).
 *  - Every call is asynchronous on the given stream.  Two entry points fork
 *    work onto a second stream and join it back with events created per call:
 *    cx_psf_4f_to_host (the caller's copy stream) and cx_multislice_backward
 *    (a stream the library creates once per device).
 */
#ifndef CX_B200_H
#define CX_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef void* cx_stream_t; /* a cudaStream_t */

typedef enum {
  CX_OK = 0,
  CX_ERR_INVALID = 1,     /* bad argument (shape, pointer, parameter) */
  CX_ERR_UNSUPPORTED = 2, /* size/feature not compiled in */
  CX_ERR_CUDA = 3,        /* a CUDA runtime call failed */
  CX_ERR_WORKSPACE = 4,   /* workspace too small */
  CX_ERR_NOT_CONVERGED = 5
} cx_status;

typedef enum {
  CX_PREC_ACCURATE = 0, /* FP64 phase arguments reduced mod 2pi, FP32 FFT */
  CX_PREC_REF32 = 1,    /* FP32 in the reference's operation order */
  CX_PREC_SPLIT16 = 2   /* as ACCURATE, with the transforms of length 1024 / 1280 run as dense DFT
                           contractions on the tensor cores (FP16 hi + lo operands, FP32 accumulation):
                           cx_psf_4f, cx_prop2d(_ptrs) and cx_multislice_* on grids with 1024 or 1280
                           (padded) rows; other entry points and grids reject it */
} cx_precision;

typedef enum {
  CX_KERNEL_TRANSFER = 0, /* Fresnel transfer function (propagation.py:466-496) */
  CX_KERNEL_ASM = 1,      /* angular spectrum (propagation.py:499-580) */
  CX_KERNEL_EXPLICIT = 2, /* caller-supplied propagator array (propagation.py:355-393) */
  CX_KERNEL_SAS = 3       /* scalable-ASM precompensation Delta H of the padded grid (propagation.py:85-103) */
} cx_kernel_kind;

/* One output plane of a batched propagation. */
typedef struct {
  double z;          /* propagation distance */
  double wavelength; /* vacuum wavelength */
  double dy, dx;     /* sample spacing of the padded input grid */
  double shift_y, shift_x;   /* ASM output-plane shift (propagation.py:551) */
  double bl_y0, bl_x0;       /* band-limit rectangle centre (propagation.py:566) */
  double bl_hy, bl_hx;       /* band-limit rectangle half width (propagation.py:574) */
  int32_t in_plane;  /* input plane (batch * n_wv + wv) this output reads */
  int32_t h_plane;   /* plane of the explicit propagator array (CX_KERNEL_EXPLICIT) */
} cx_plane;

/* Fourier-multiplier propagation: pad -> FFT2 -> x H -> IFFT2 -> crop. */
typedef struct {
  int32_t ny, nx;          /* input spatial shape */
  int32_t pad_y, pad_x;    /* zero padding on each side */
  int32_t n_wv;            /* interleaved wavelengths (1: monochromatic layout) */
  int32_t n_in_planes;     /* input batch * n_wv */
  int32_t n_out_planes;    /* output batch * n_wv (entries in the cx_plane array) */
  int32_t mode_same;       /* 1: crop the output back to ny x nx */
  int32_t kernel;          /* cx_kernel_kind */
  int32_t precision;       /* cx_precision */
  int32_t remove_evanescent;
  int32_t bandlimit;
  double n_medium;
  double ky0, kx0;         /* kykx tilt subtracted from the frequency grid */
  int32_t conj_kernel;     /* 1: multiply by conj(H) instead of H -- the adjoint of the propagation
                              (conj(H) = H(-z) for the transfer and ASM kernels, all options included) */
  int32_t crop_y, crop_x;  /* mode_same = 0 only: rows / columns dropped on each side of the padded grid
                              (the adjoint of zero padding); output (py - 2 crop_y, px - 2 crop_x) */
  int32_t reserved;
} cx_prop2d_desc;

/* Workspace bytes for cx_prop2d. */
cx_status cx_prop2d_workspace_size(const cx_prop2d_desc* d, size_t* bytes);

/* transfer_propagate / asm_propagate / kernel_propagate (FFT branch)
 * (functional/propagation.py:168-252, 255-352, 355-394).
 * u_out: (n_out_planes/n_wv, oy, ox, n_wv) with (oy, ox) = (ny, nx) when
 * mode_same else (ny + 2 pad_y - 2 crop_y, nx + 2 pad_x - 2 crop_x).
 * The gradient of a propagation (the reference differentiates it with
 * jax.grad) is the same call with conj_kernel = 1 applied to the output
 * gradient: mode_same keeps its geometry; a "full" propagation's adjoint takes
 * the padded grid as input (pad 0) and crops (pad_y, pad_x).  H (CX_KERNEL_EXPLICIT only):
 * planar (h_planes, py, px) complex64 in FFT (ifftshifted) order. */
cx_status cx_prop2d(const cx_prop2d_desc* d, const cx_plane* planes_dev, const void* u_in, void* u_out,
                    const void* H, void* workspace, size_t workspace_bytes, cx_stream_t stream);

/* cx_prop2d over a batch of fields at independent addresses: element b of the
 * input batch (ny, nx, n_wv interleaved) starts at u_in_ptrs_dev[b], element b
 * of the output batch at u_out_ptrs_dev[b]; both arrays live in DEVICE
 * memory, with n_in_planes / n_wv and n_out_planes / n_wv entries.  The
 * planes' in_plane indices refer to positions in the input batch.  Used by
 * the continuous-batching server, whose requests own separate buffers.  No
 * counterpart in the reference (jax batches through vmap). */
cx_status cx_prop2d_ptrs(const cx_prop2d_desc* d, const cx_plane* planes_dev, const void* const* u_in_ptrs_dev,
                         void* const* u_out_ptrs_dev, const void* H, void* workspace, size_t workspace_bytes,
                         cx_stream_t stream);

/* compute_transfer_propagator / compute_asm_propagator
 * (functional/propagation.py:466-496, 499-580): writes the ifftshifted
 * propagator, planar (n_out_planes, py, px) complex64, py/px = padded size. */
cx_status cx_fill_propagator(const cx_prop2d_desc* d, const cx_plane* planes_dev, void* H_out,
                             cx_stream_t stream);

/* ---------------------------------------------------------------------------
 * Batched 4f widefield PSF:
 *   objective_point_source (functional/sources.py:122-209)
 *   -> phase_change (functional/phase_masks.py:29-68)
 *   -> ff_lens (functional/lenses.py:64-95 via convenience.py:9-59)
 *   -> Field.intensity (core/field.py:735-740)
 * fused: the source, pupil, power normalisation, phase mask and lens
 * normalisation are evaluated inside the FFT loader; the fftshifts are index
 * remaps; the spectral sum of |u|^2 is the FFT epilogue.
 * ------------------------------------------------------------------------- */
typedef struct {
  int32_t ny, nx;        /* grid */
  int32_t n_z;           /* defocus planes */
  int32_t n_wv;          /* wavelengths */
  int32_t precision;     /* cx_precision */
  int32_t has_phase;     /* phase mask present */
  int32_t spectrally_modulate;
  int32_t normalize_power; /* objective_point_source(power=...) not None */
  double f_obj, n_medium, NA, power;
  double amplitude;      /* scalar source amplitude */
  double offset_y, offset_x;
  double f_lens;         /* ff_lens focal length (negative: inverse lens) */
  double lens_NA;        /* ff_lens pupil NA, <= 0: none */
} cx_psf_desc;

/* Per-wavelength parameters of the PSF (host memory, n_wv entries each). */
typedef struct {
  const double* wavelength; /* n_wv */
  const double* density;    /* n_wv, normalised spectral density */
  const double* dy;         /* n_wv source spacing y */
  const double* dx;         /* n_wv source spacing x */
} cx_psf_spectrum;

cx_status cx_psf_workspace_size(const cx_psf_desc* d, size_t* bytes);

/* z_dev: n_z defocus distances (device, double).  phase: (ny, nx) float32 or
 * NULL.  intensity_out: (n_z, ny, nx) float32. */
cx_status cx_psf_4f(const cx_psf_desc* d, const cx_psf_spectrum* spec, const double* z_dev, const float* phase,
                    float* intensity_out, void* workspace, size_t workspace_bytes, cx_stream_t stream);

/* Chunking of cx_psf_4f: info[0] = z planes per chunk, info[1] = stored rows
 * per plane stack (pupil rows of all wavelengths), info[2] = number of chunks. */
cx_status cx_psf_plan_info(const cx_psf_desc* d, const cx_psf_spectrum* spec, int32_t* info);

/* The PSF stack of cx_psf_4f written into HOST memory (n_z x ny x nx
 * float32 at intensity_host).  Groups of z-planes are computed on `stream`
 * into a ring of device slots inside the workspace, and each group's copy to
 * the host runs on `copy_stream` while later groups compute, so the transfer
 * overlaps the FFTs (intensity_host must be page-locked for that; pageable
 * memory works without overlap).  Everything is ordered before later work on
 * `stream`.  No counterpart in the reference (XLA decides its transfers).
 * Workspace: cx_psf_host_workspace_size. */
cx_status cx_psf_host_workspace_size(const cx_psf_desc* d, const cx_psf_spectrum* spec, size_t* bytes);
cx_status cx_psf_4f_to_host(const cx_psf_desc* d, const cx_psf_spectrum* spec, const double* z_dev,
                            const float* phase, float* intensity_host, void* workspace, size_t workspace_bytes,
                            cx_stream_t stream, cx_stream_t copy_stream);

/* One stage of cx_psf_4f, for measuring kernels in isolation: stage -1 =
 * pupil counts (must run first), 0 = row pass of `chunk`, 1 = column pass of
 * `chunk`.  Same arguments as cx_psf_4f. */
cx_status cx_psf_4f_stage(const cx_psf_desc* d, const cx_psf_spectrum* spec, const double* z_dev, const float* phase,
                          float* intensity_out, void* workspace, size_t workspace_bytes, int32_t stage,
                          int32_t chunk, cx_stream_t stream);

/* objective_point_source [-> phase_change] materialised
 * (functional/sources.py:122-209, functional/phase_masks.py:29-68):
 * u_out (n_z, ny, nx, n_wv) complex64, power-normalised; f_lens / lens_NA are
 * ignored.  workspace: >= 256 bytes. */
cx_status cx_psf_source(const cx_psf_desc* d, const cx_psf_spectrum* spec, const double* z_dev, const float* phase,
                        void* u_out, void* workspace, size_t workspace_bytes, cx_stream_t stream);

/* ---------------------------------------------------------------------------
 * Centred optical FFT with fused chirps
 *   optical_fft        functional/convenience.py:9-59 (+ utils/fft.py:8-20)
 *   ff_lens / df_lens  functional/lenses.py:64-95, 159-198
 *   transform_propagate functional/propagation.py:34-82
 * out = crop( post * chirp_out * C( FFT2_shifted( pre * C(pad(u) * chirp_in * pupil) ) ) )
 * with C = complex conjugation when `conj` is set (the z < 0 branch of
 * optical_fft), FFT2_shifted = fftshift(fft2(ifftshift(.))) done by index
 * remapping, chirp_* = exp(i c |r|^2) on the input / output grid.
 * ------------------------------------------------------------------------- */
typedef struct {
  double pre_re, pre_im;   /* complex factor on the (conjugated) input */
  double post_re, post_im; /* complex factor on the (conjugated) output */
  double chirp_in;         /* input phase coefficient c_in (0: none) */
  double chirp_out;        /* output phase coefficient c_out (0: none) */
  double dy_in, dx_in;     /* input grid spacing (padded grid) */
  double dy_out, dx_out;   /* output grid spacing */
  double oy, ox;           /* grid origin */
  double pupil_r2;         /* circular input pupil radius^2 (< 0: none) */
  int32_t in_plane;        /* input plane (batch * n_wv + wv) */
  int32_t conj;            /* 1: conjugate input and output (inverse transform) */
  double pupil_out_r2;     /* > 0: circular pupil of this radius^2 on the output grid (origin oy, ox), applied
                              last; <= 0: none.  The adjoint of an input pupil. */
} cx_fft_plane;

typedef struct {
  int32_t ny, nx;          /* input spatial shape */
  int32_t pad_y, pad_x;    /* zero padding on each side before the transform */
  int32_t crop_y, crop_x;  /* crop on each side after the transform */
  int32_t n_wv;            /* interleaved wavelengths of input and output */
  int32_t n_in_planes, n_out_planes;
  int32_t precision;       /* cx_precision */
} cx_optfft_desc;

cx_status cx_optfft_workspace_size(const cx_optfft_desc* d, size_t* bytes);
/* planes_dev: n_out_planes cx_fft_plane in device memory.  u_out:
 * (n_out_planes/n_wv, ny + 2 pad_y - 2 crop_y, nx + 2 pad_x - 2 crop_x, n_wv).
 * Adjoint (the gradient jax.grad takes through optical_fft / ff_lens): the
 * same call on the output gradient with pad and crop swapped, spacings
 * swapped, conj flipped, chirp_in' = -chirp_out, chirp_out' = -chirp_in,
 * pre' = post (conj = 0 forward) or conj(post) (conj = 1), post' = conj(pre)
 * or pre, and the input pupil moved to pupil_out_r2. */
cx_status cx_optical_fft(const cx_optfft_desc* d, const cx_fft_plane* planes_dev, const void* u_in, void* u_out,
                         void* workspace, size_t workspace_bytes, cx_stream_t stream);
/* Same, with a propagator table H (planar (n_out_planes, py, px), FFT order)
 * multiplied into the spectrum before the fftshift: with pre = post = 1 this
 * is fftshift(H * fft2(ifftshift(pad(u)))), the spectrum the CZT branch of
 * kernel_propagate starts from (functional/propagation.py:414-418). */
cx_status cx_optical_fft_h(const cx_optfft_desc* d, const cx_fft_plane* planes_dev, const void* H, const void* u_in,
                           void* u_out, void* workspace, size_t workspace_bytes, cx_stream_t stream);

/* ---------------------------------------------------------------------------
 * Thick-sample multislice, forward and adjoint
 *   multislice_thick_sample (functional/samples.py:137-282) with
 *   thin_sample (samples.py:85-134) and the ASM kernel (propagation.py:499-580)
 * u_{i+1} = t_i * IFFT2(H(dz) FFT2(u_i)), t_i = exp(i 2 pi dz/lambda (dn_i + i abs_i)),
 * then the defocus by -reverse_distance (ASM, optional NA mask) and the crop.
 * The adjoint takes g_out = dL/dRe(u_out) + i dL/dIm(u_out) and returns
 * dL/d dn, dL/d abs (and dL/du_in), recomputing each checkpoint segment (the
 * next segment's recomputation runs on a library-owned second stream of the
 * current device, joined back into `stream` by events before the call's last
 * launch; the workspace holds two segments of records).
 * ------------------------------------------------------------------------- */
typedef struct {
  int32_t ny, nx;            /* field shape (unpadded) */
  int32_t pad;               /* pad_width on each side */
  int32_t n_slices;          /* D */
  int32_t precision;         /* cx_precision */
  int32_t remove_evanescent, bandlimit;  /* slice propagator options */
  int32_t checkpoint_every;  /* K; <= 0: ceil(sqrt(D)) */
  double n_medium, wavelength, dy, dx;
  double dz;                 /* thickness_per_slice */
  double reverse_distance;   /* defocus back by this distance */
  double NA;                 /* <= 0: no NA mask */
  double ky0, kx0;           /* kykx */
} cx_ms_desc;

cx_status cx_multislice_workspace_size(const cx_ms_desc* d, int32_t need_grad, size_t* bytes);
/* number of planes the forward writes into `checkpoints` (each (ny + 2 pad) x (nx + 2 pad) complex64):
 * one every K slices, then the fields after each slice of the last segment (which the adjoint
 * therefore does not recompute) */
int32_t cx_multislice_num_checkpoints(const cx_ms_desc* d);
/* dn, abs: (D, ny, nx) float32; u_in, u_out: (ny, nx) complex64; checkpoints may be NULL
 * (forward only). */
cx_status cx_multislice_forward(const cx_ms_desc* d, const void* u_in, const float* dn, const float* abs_,
                                void* u_out, void* checkpoints, void* workspace, size_t workspace_bytes,
                                cx_stream_t stream);
cx_status cx_multislice_backward(const cx_ms_desc* d, const float* dn, const float* abs_, const void* checkpoints,
                                 const void* grad_out, float* grad_dn, float* grad_abs, void* grad_u_in,
                                 void* workspace, size_t workspace_bytes, cx_stream_t stream);

/* ---------------------------------------------------------------------------
 * Chirp-Z transform along one axis (Bluestein)
 *   czt / cztn / zoomed_fft (utils/czt.py:7-124) and the CZT branch of
 *   kernel_propagate (functional/propagation.py:420-443)
 * y[k] = scale [w^(-N k) a^N] sum_j x[j] a^(-j) w^(j k),  k < m
 * Vectors v = o * inner + i; element j of vector v at
 * x + o*in_ostride + i*in_istride + j*in_estride (likewise for y, k).
 * ------------------------------------------------------------------------- */
typedef struct {
  int32_t n, m;        /* input / output length */
  int32_t L;           /* FFT length >= n + m - 1 (0: smallest compiled length) */
  int32_t inner;       /* vectors per outer index */
  int64_t n_vec;
  int64_t in_ostride, in_istride, in_estride;
  int64_t out_ostride, out_istride, out_estride;
  double a_re, a_im, w_re, w_im;
  int32_t mod_n;       /* >= 0: multiply output k by w^(-mod_n k) a^mod_n */
  int32_t layout;      /* 0: one team per vector; 1: column tiles (unit inner strides) */
  double scale;
  int32_t adjoint;     /* 1: the adjoint (conjugate transpose) of the transform above:
                          x'[j] = sum_k conj(scale [w^(-N k) a^N] a^(-j) w^(j k)) y'[k], j < n.
                          Input vectors then have m elements and outputs n (strides as given). */
  int32_t reserved;
} cx_czt_desc;

cx_status cx_czt_workspace_size(const cx_czt_desc* d, size_t* bytes);
cx_status cx_czt(const cx_czt_desc* d, const void* x, void* y, void* workspace, size_t workspace_bytes,
                 cx_stream_t stream);

/* cx_czt without a workspace argument; allocates no device memory.  No
 * counterpart in the reference: its czt (utils/czt.py:7-52) is a traced JAX
 * function whose temporaries XLA places.  This entry point is for callers that
 * can neither allocate device memory nor hand out scratch, e.g. a
 * foreign-function handler running under a framework that owns the whole
 * device pool and offers no allocator for temporaries.
 *  - The chirp filter and its spectrum live in one static 64 KiB device
 *    buffer inside the library: FFT lengths L <= 4096 (n + m - 1 <= 4096);
 *    larger requests return CX_ERR_UNSUPPORTED with a message.
 *  - The first call on each device (with that device current) uploads the
 *    twiddle table and looks up the buffer's address with synchronous runtime
 *    calls; make that first call (or cx_init plus one call) before any stream
 *    capture begins.
 *  - Every call on a device uses the same buffer: calls that can overlap in
 *    time (streams without ordering between them, several host threads)
 *    race on it and must be serialised by the caller.
 *  - Results are identical to cx_czt's for the same descriptor and input. */
cx_status cx_czt_noalloc(const cx_czt_desc* d, const void* x, void* y, cx_stream_t stream);

/* Rescaled-output propagation in one call: the CZT branch of kernel_propagate
 * (functional/propagation.py:395-443) as reached from transfer_propagate /
 * asm_propagate with output_dx / output_shape (:168-352): propagator of the
 * padded grid, fftshift(H fft2(ifftshift(pad u))), then a chirp-Z transform
 * along y and along x onto the (my, mx) output grid of spacing (dy_out,
 * dx_out) shifted by (shift_y, shift_x).  n_fields single-wavelength fields
 * (ny, nx) complex64 sharing every parameter; u_out (n_fields, my, mx).
 * bandlimit = 1 applies the Matsushima band-limit rectangle bl_* to the ASM
 * propagator (the caller computes it, e.g. as _bandlimit_rect does).
 * method 1 replaces the two CZTs by the Yu et al. rescaled convolution:
 * fftconvolve(B, f, "same") of the chirped spectrum with a chirp filter,
 * separable per axis, times the output chirp; shift_y/x is the output
 * grid origin there. */
typedef struct {
  int32_t ny, nx;          /* input shape */
  int32_t pad_y, pad_x;    /* zero padding on each side */
  int32_t my, mx;          /* output shape (>= 2 each) */
  int32_t n_fields;
  int32_t kernel;          /* CX_KERNEL_TRANSFER or CX_KERNEL_ASM */
  int32_t precision;       /* cx_precision */
  int32_t remove_evanescent, bandlimit;
  int32_t method;          /* 0: chirp-Z transforms (use_czt=True); 1: the Yu et al. chirp convolution
                              (use_czt=False, propagation.py:445-458; output shape = padded shape) */
  double n_medium, z, wavelength;
  double dy_in, dx_in, dy_out, dx_out;
  double shift_y, shift_x;
  double ky0, kx0;
  double bl_y0, bl_x0, bl_hy, bl_hx; /* band-limit rectangle (bandlimit = 1, ASM only; as in cx_plane) */
} cx_czt_prop_desc;

cx_status cx_czt_propagate_workspace_size(const cx_czt_prop_desc* d, size_t* bytes);
cx_status cx_czt_propagate(const cx_czt_prop_desc* d, const void* u_in, void* u_out, void* workspace,
                           size_t workspace_bytes, cx_stream_t stream);

/* ---------------------------------------------------------------------------
 * Fluorescent thick sample: fluorescent_multislice_thick_sample
 * (functional/samples.py:285-441).  Per Monte-Carlo sample: the padded field
 * goes through D slices, u <- IFFT2(FFT2(u exp(i 2 pi dz dn_i / lambda)
 * + fl_i exp(i ph_i)) H(dz)) (ASM, band limit / evanescent options as
 * compute_asm_propagator), then out[D - 1 - i] += |crop(IFFT2(U H(-dz)^(i+1)))|^2
 * with U = FFT2(u_D); the next sample starts from U H(-dz)^D, as the
 * reference's loop carries it; out is divided by num_samples.
 * u_in: (ny, nx) complex64; fluorescence, dn: (D, ny, nx) float32;
 * phases: (num_samples, D, ny, nx) float32 in radians, or NULL: phase =
 * float32(2 pi) * (top 24 bits of splitmix64(seed + (c + 1) * 0x9E3779B97F4A7C15)) / 2^24,
 * c = sample * D ny nx + (i ny + y) nx + x (the reference draws them from
 * jax.random, which this library does not reproduce); out: (D, ny, nx) float32.
 * ------------------------------------------------------------------------- */
typedef struct {
  int32_t ny, nx;            /* field shape (unpadded) */
  int32_t pad;               /* pad_width on each side */
  int32_t n_slices;          /* D */
  int32_t num_samples;       /* Monte-Carlo samples */
  int32_t remove_evanescent, bandlimit;
  int32_t reserved;
  uint64_t seed;             /* phase generator seed (phases == NULL) */
  double n_medium, wavelength, dy, dx;
  double dz;                 /* thickness_per_slice */
  double ky0, kx0;           /* kykx */
} cx_fluor_desc;

cx_status cx_fluorescent_multislice_workspace_size(const cx_fluor_desc* d, size_t* bytes);
cx_status cx_fluorescent_multislice(const cx_fluor_desc* d, const void* u_in, const float* fluorescence,
                                    const float* dn, const float* phases, float* out, void* workspace,
                                    size_t workspace_bytes, cx_stream_t stream);

/* ---------------------------------------------------------------------------
 * Ray transfer: ray_transfer (functional/rays.py:102-154), Collins' integral
 * of an ABCD system with magnification M:
 *   u_out = exp(i k (D - 1/M) |g|^2 / (2B M^4)) IFFT2(H FFT2(exp(i k (A - M) |g|^2 / (2B)) u_in)),
 * H = exp(-i pi (lambda / n) (B / M) |f|^2) (the transfer kernel of z = B/M),
 * g = (i - N/2) d + origin, k = 2 pi n / lambda; the output spacing is d / M
 * (the caller's metadata).  u_in, u_out: (batch, ny, nx, n_wv) complex64
 * (n_wv = 1: (batch, ny, nx)); planes_dev: n_planes = batch * n_wv cx_plane
 * entries (wavelength, dy, dx of each plane; z is set to B / M inside).
 * ------------------------------------------------------------------------- */
typedef struct {
  int32_t ny, nx, n_wv;
  int32_t n_planes;        /* batch * n_wv */
  int32_t precision;       /* cx_precision of the transfer kernel */
  int32_t reserved;
  double A, B, D;          /* ABCD[0][0], ABCD[0][1], ABCD[1][1] */
  double magnification;
  double n_medium;
  double origin_y, origin_x;
} cx_ray_desc;

cx_status cx_ray_transfer_workspace_size(const cx_ray_desc* d, size_t* bytes);
cx_status cx_ray_transfer(const cx_ray_desc* d, const cx_plane* planes_dev, const void* u_in, void* u_out,
                          void* workspace, size_t workspace_bytes, cx_stream_t stream);

/* ---------------------------------------------------------------------------
 * Polarized thick sample: polarized_multislice_thick_sample
 * (functional/samples.py:444-546) of a vector field u_in (ny, nx, 3)
 * complex64, components (z, y, x) -- or of one wavelength of a chromatic
 * vector field (ny, nx, n_wv, 3) -- through D slices of a real
 * scattering potential (D, ny, nx, 3, 3) float32 (rows and columns in
 * (z, y, x) order), on the grid zero-padded to (2 ny, 2 nx):
 *   u <- crop IFFT2(Q (e FFT2(pad u) + h FFT2(pad(V_i crop IFFT2(Q FFT2(pad u))))))
 * Q = I - k k^T / km^2 (k = (kz, ky, kx), km = 2 pi n / lambda, zero where
 * |k_perp| > NA km), e = exp(i kz dz), h = -i/2 exp(i kz dz) dz / kz (0 where
 * kz = 0).  Even ny, nx (the reference takes its frequencies from the field
 * padded by N // 2 per side, which is 2N only for even N), 2N <= 4096.
 * ------------------------------------------------------------------------- */
typedef struct {
  int32_t ny, nx;
  int32_t n_slices;
  int32_t n_wv, wv;        /* u is (ny, nx, n_wv, 3); this call processes wavelength wv (the reference
                              broadcasts the potential over the wavelengths of a chromatic field) */
  int32_t reserved;
  double n_medium, wavelength, dy, dx;  /* of wavelength wv */
  double dz;               /* thickness_per_slice */
  double NA;
} cx_polar_desc;

cx_status cx_polarized_multislice_workspace_size(const cx_polar_desc* d, size_t* bytes);
cx_status cx_polarized_multislice(const cx_polar_desc* d, const void* u_in, const float* potential, void* u_out,
                                  void* workspace, size_t workspace_bytes, cx_stream_t stream);

/* ---------------------------------------------------------------------------
 * High-NA lens: high_na_ff_lens (functional/lenses.py:98-156) of n_fields
 * monochromatic fields (ny, nx) complex64, scalar, or vectorial (ny, nx, 3)
 * with components (z, y, x) converted to the spherical basis first
 * (cartesian_to_spherical, core/field.py:897-940).  The defocus
 * exp(i k sz f) / sz on the pupil's frequency grid (k = 2 pi n / lambda,
 * sz = sqrt(max(1 - NA^2 |f_grid lambda / n|^2, 0)), 0 where sz = 0), then the
 * zoomed FFT over [-zoom pi, zoom pi] with the end point onto (my, mx),
 * zoom = 2 NA my output_dx / ((nx - 1) lambda).  u_out: (n_fields, my, mx[, 3]).
 * ------------------------------------------------------------------------- */
typedef struct {
  int32_t n_fields;
  int32_t ny, nx;          /* pupil grid (nx >= 2) */
  int32_t my, mx;          /* output grid (>= 2 each) */
  int32_t vectorial;       /* 0: scalar; 1: vector field, 3 components innermost */
  double f, n_medium, NA, wavelength;
  double dy, dx;           /* pupil spacing */
  double origin_y, origin_x; /* pupil grid origin (vector basis change) */
  double output_dx;        /* output pixel pitch (both axes) */
} cx_high_na_desc;

cx_status cx_high_na_ff_lens_workspace_size(const cx_high_na_desc* d, size_t* bytes);
cx_status cx_high_na_ff_lens(const cx_high_na_desc* d, const void* u_in, void* u_out, void* workspace,
                             size_t workspace_bytes, cx_stream_t stream);

/* ---------------------------------------------------------------------------
 * Incoherent imaging: fourier_convolution (ops/ops.py:9-86, axes (-2, -1),
 * mode "same") of a sample stack with a kernel (PSF) stack, plane by plane,
 * and the sensor's sum over the planes (functional/sensors.py:85-86,
 * systems/microscopes.py:271-297).  sample: (n_planes, h, w) float32;
 * kernel: (n_planes, kh, kw) float32, or one (kh, kw) plane for all planes
 * (kernel_broadcast = 1); out: (h, w) float32 if reduce, else
 * (n_planes, h, w), cropped from offset ((kh - 1) / 2, (kw - 1) / 2) of the
 * full convolution.  Any transform size >= h + kh - 1 by w + kw - 1 gives
 * the same linear convolution after the crop: the smallest supported even
 * lengths >= 2 max(h, kh), 2 max(w, kw) are used (2..4096 per axis), or the
 * smallest powers of two >= those with pow2_lengths = 1.
 * ------------------------------------------------------------------------- */
typedef struct {
  int32_t n_planes, h, w;
  int32_t kh, kw;
  int32_t kernel_broadcast; /* 1: one (kh, kw) kernel for every plane */
  int32_t reduce;           /* 1: sum over the planes (BasicSensor(reduce_axis=0)) */
  int32_t pow2_lengths;     /* 1: transform lengths are powers of two */
} cx_conv_desc;

cx_status cx_conv2d_workspace_size(const cx_conv_desc* d, size_t* bytes);
cx_status cx_conv2d_same(const cx_conv_desc* d, const float* sample, const float* kernel, float* out, void* workspace,
                         size_t workspace_bytes, cx_stream_t stream);

/* ---------------------------------------------------------------------------
 * Modified Born series (experimental/modified_born_series/solver.py:42-146)
 * Grid (X, Y, Z); fields are three component planes (3, X, Y, Z) complex64;
 * eps (X, Y, Z) complex64.  s = 1 / (1.1 i R) and kb2 = shift * s + 1 are the
 * preconditioner's scale and k_bias^2 (solver.py:64-65).
 * ------------------------------------------------------------------------- */
typedef struct {
  int32_t X, Y, Z;
  double spacing, k0;
  double s_re, s_im, kb2_re, kb2_im;
} cx_mbs_desc;

cx_status cx_mbs_workspace_size(const cx_mbs_desc* d, size_t* bytes);
/* prec_y = -V(G(s * src)) (solver.py:87-96, before the num_scale division) */
cx_status cx_mbs_precondition(const cx_mbs_desc* d, const void* eps, const void* src, void* prec_y, void* workspace,
                              size_t workspace_bytes, cx_stream_t stream);
/* x_new = prec_y - prec_forward(x) + x (solver.py:91-93, 136-142);
 * acc (device, 2 doubles) = (sum |x_new - x|^2, sum |x_new|^2), FP64. */
cx_status cx_mbs_iterate(const cx_mbs_desc* d, const void* eps, const void* prec_y, const void* x, void* x_new,
                         double* acc, void* workspace, size_t workspace_bytes, cx_stream_t stream);

/* prec_forward(x) = -V(G(V x) + x) (solver.py:91-93): the preconditioned
 * operator whose system prec_forward(x) = prec_y BiCGStab solves
 * (solver.py:143-144, jax.scipy.sparse.linalg.bicgstab). */
cx_status cx_mbs_forward(const cx_mbs_desc* d, const void* eps, const void* x, void* out, void* workspace,
                         size_t workspace_bytes, cx_stream_t stream);

/* Complex vector algebra for the Krylov solve, FP64 accumulation (the
 * reference's bicgstab takes these inner products in its working precision):
 * out_dev[0..3] = (Re, Im) sum conj(x) y, sum |x|^2, sum |y|^2 over n complex64. */
cx_status cx_cvec_dot(const void* x, const void* y, int64_t n, double* out_dev, cx_stream_t stream);
/* out = c0 x + c1 y [+ c2 z] with complex coefficients coef (host, 6 doubles:
 * re, im of c0, c1, c2; z may be NULL); norm_dev (may be NULL) = sum |out|^2. */
cx_status cx_cvec_lincomb(int64_t n, const double* coef, const void* x, const void* y, const void* z, void* out,
                          double* norm_dev, cx_stream_t stream);

/* Field.intensity (core/field.py:656-665, 735-740): out[b, y, x] =
 * sum_wv density[wv] |u[b, y, x, wv]|^2.  density_dev: n_wv doubles. */
cx_status cx_intensity(const void* u, int64_t n_pix, int32_t n_wv, const double* density_dev, float* out,
                       cx_stream_t stream);

/* ---------------------------------------------------------------------------
 * Elementwise field operations and the adjoints jax.grad takes through them.
 * u, out: (n_batch, ny, nx, n_wv) complex64 (n_wv interleaved innermost:
 * wavelengths, or wavelengths x vector components); real maps: one (ny, nx)
 * float32 plane broadcast over batch and channels, or (n_batch, ny, nx) when
 * map_batched = 1.  Gradients follow torch's convention for complex values
 * (g = dL/dRe + i dL/dIm); the gradient of a broadcast map is summed over
 * batch and channels.
 * ------------------------------------------------------------------------- */
typedef struct {
  int64_t n_batch;
  int32_t ny, nx;
  int32_t n_wv;          /* interleaved innermost channels, 1..64 */
  int32_t map_batched;   /* 1: the real maps have n_batch planes */
} cx_ew_desc;

/* phase_change (functional/phase_masks.py:29-68): out = u exp(i phase s[w]),
 * s (device, n_wv floats) = lambda0 / lambda_w (spectrally_modulate) or 1. */
cx_status cx_phase_change(const cx_ew_desc* d, const void* u, const float* phase, const float* s_dev, void* out,
                          cx_stream_t stream);
/* Its adjoint: g_u = g exp(-i phase s[w]); g_phase = sum_{b,w} s[w] Im(g conj(out)).
 * g_u or g_phase may be NULL (not wanted). */
cx_status cx_phase_change_adjoint(const cx_ew_desc* d, const void* g, const void* out, const float* phase,
                                  const float* s_dev, void* g_u, float* g_phase, cx_stream_t stream);
/* thin_sample (functional/samples.py:85-134): out = u exp(i kd[w] (dn + i absorption)),
 * kd (device, n_wv floats) = 2 pi thickness / lambda_w. */
cx_status cx_thin_sample(const cx_ew_desc* d, const void* u, const float* absorption, const float* dn,
                         const float* kd_dev, void* out, cx_stream_t stream);
/* Its adjoint: g_u = g conj(t); g_dn = sum kd Im(g conj(out)); g_absorption = -sum kd Re(g conj(out)). */
cx_status cx_thin_sample_adjoint(const cx_ew_desc* d, const void* g, const void* out, const float* absorption,
                                 const float* dn, const float* kd_dev, void* g_u, float* g_absorption, float* g_dn,
                                 cx_stream_t stream);
/* Adjoint of Field.intensity (core/field.py:656-665, 735-740):
 * g_u[p, w] = 2 density[w] g_intensity[p] u[p, w]. */
cx_status cx_intensity_adjoint(const void* u, int64_t n_pix, int32_t n_wv, const double* density_dev,
                               const float* g_intensity, void* g_u, cx_stream_t stream);
/* pad (core/field.py:534-549) of the spatial axes with the constant cval:
 * out (n_batch, ny + 2 pad_y, nx + 2 pad_x, n_wv). */
cx_status cx_pad(const cx_ew_desc* d, int32_t pad_y, int32_t pad_x, float cval_re, float cval_im, const void* u,
                 void* out, cx_stream_t stream);
/* plane_wave (functional/sources.py:212-293) before its pupil and power
 * normalisation: u[b, y, x, w] = amp_w exp(i (ky gy + kx gx)), g = d_w (i - N/2)
 * + origin; wv_params_dev: (n_wv, 3) doubles (dy, dx, amp). */
cx_status cx_plane_wave(const cx_ew_desc* d, const double* wv_params_dev, double ky, double kx, double origin_y,
                        double origin_x, void* u, cx_stream_t stream);
/* The Fourier multiplier of kernel_propagate (functional/propagation.py:391-394)
 * for grids the fused passes do not cover (their transforms are chirp-Z passes):
 * out[b, y, x, w] = u[b, y, x, w] H[b n_wv + w, y, x], conj(H) when conj_h; H
 * planar (n_batch n_wv, ny, nx) as cx_fill_propagator writes it. */
cx_status cx_cmul_planar(const cx_ew_desc* d, const void* u, const void* H, int32_t conj_h, void* out,
                         cx_stream_t stream);
/* Pupils (functional/pupils.py:17-67) on the field grid g = d_w (i - N/2) + origin:
 * kind 0 circular (|g|^2 <= p0^2), 1 square (max |g| <= p0), 2 super-Gaussian
 * exp(-(|g| / p0)^p1), 3 Tukey (alpha p1 on |g / extent|, extent (p2, p3));
 * wv_params_dev: (n_wv, 6) doubles (dy, dx, p0, p1, p2, p3).  out = mask * u. */
cx_status cx_pupil(const cx_ew_desc* d, int32_t kind, const double* wv_params_dev, double origin_y, double origin_x,
                   const void* u, void* out, cx_stream_t stream);

/* ---------------------------------------------------------------------------
 * Tensor-core (tcgen05) split-precision DFT: the building block of the
 * CX_PREC_SPLIT16 transform stages that replace the radix butterflies of
 * the FFTs inside kernel_propagate (functional/propagation.py:391-394) and
 * optical_fft (functional/convenience.py:9-59).  y[b, k] = sum_n x[b, n]
 * exp(-+2 pi i n k / R) for R in {16, 32, 40, 64}, x, y (batch, R) complex64:
 * a real GEMM on FP16 hi + lo operands (3 products, FP32 accumulation in
 * tensor memory), each vector scaled by a power of two.  status_dev[0] is
 * set to 1 if the kernel gave up waiting for an MMA (the output is then
 * incomplete).
 * ------------------------------------------------------------------------- */
cx_status cx_dft_split16(const void* x, void* y, int32_t R, int64_t batch, int32_t inverse, int32_t* status_dev,
                         cx_stream_t stream);

/* Number of CTAs of the CX_PREC_SPLIT16 PSF / propagation / multislice
 * kernels that gave up waiting for a tensor-core MMA on the current device
 * since the last reset (their output tiles are then NaN).  Synchronises the
 * device; reset != 0 clears the count after reading it. */
cx_status cx_tc_timeouts(int32_t* count, int32_t reset);

/* ---------------------------------------------------------------------------
 * misc
 * ------------------------------------------------------------------------- */
const char* cx_last_error(void);
int32_t cx_version(void);
/* One-time set-up of the current device (uploads the FFT twiddle tables).
 * Every entry point does this on its first call on a device; call cx_init
 * explicitly before capturing a stream into a CUDA graph. */
cx_status cx_init(void);
/* 1 if an FFT length is compiled in (fast path), else 0. */
int32_t cx_fft_size_supported(int32_t n);
/* Batched complex FFT along the last axis (test/utility entry):
 * in/out (batch, n) complex64, inverse=1 applies exp(+i..) and 1/n. */
cx_status cx_fft1d(const void* in, void* out, int32_t n, int64_t batch, int32_t inverse, cx_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* CX_B200_H */
