"""Tensor-core (tcgen05) split-FP16 DFT against an FP64 DFT.

The transform is a real GEMM on FP16 hi + lo operands with FP32 accumulation;
its relative L2 error per vector is bounded by ~2^-21 times a small factor,
so the bar is 1e-5 (the accurate mode's), checked per vector over inputs
whose magnitudes span 1e-4 .. 1e4 (each vector is scaled by a power of two
before the split)."""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _lib():
    from chromatix_b200 import _native as nat

    L = nat.lib()
    L.cx_dft_split16.restype = ctypes.c_int32
    L.cx_dft_split16.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_int32,
                                 ctypes.c_void_p, ctypes.c_void_p]
    return nat, L


@pytest.mark.parametrize("R", [16, 32, 40, 64])
@pytest.mark.parametrize("inverse", [0, 1])
def test_split16_dft_matches_fp64(R, inverse):
    import torch

    nat, L = _lib()
    rng = np.random.default_rng(R + 100 * inverse)
    B = 1000  # not a multiple of the 128-vector tile
    mag = 10.0 ** rng.uniform(-4, 4, (B, 1))
    x = ((rng.standard_normal((B, R)) + 1j * rng.standard_normal((B, R))) * mag).astype(np.complex64)
    x[7] = 0  # an all-zero vector
    xt = torch.as_tensor(x, device="cuda")
    yt = torch.full_like(xt, float("nan"))
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    nat.check(L.cx_dft_split16(xt.data_ptr(), yt.data_ptr(), R, B, inverse, status.data_ptr(),
                               torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    y = yt.cpu().numpy()
    ref = np.fft.ifft(x.astype(np.complex128), axis=1) * R if inverse else np.fft.fft(x.astype(np.complex128), axis=1)
    num = np.linalg.norm(y - ref, axis=1)
    den = np.linalg.norm(ref, axis=1)
    assert np.all(y[7] == 0)
    ok = den > 0
    err = num[ok] / den[ok]
    assert err.max() < 1e-5, err.max()


def test_split16_rejects_unsupported_length():
    import torch

    nat, L = _lib()
    xt = torch.zeros((4, 24), dtype=torch.complex64, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert L.cx_dft_split16(xt.data_ptr(), xt.data_ptr(), 24, 4, 0, status.data_ptr(), None) == nat.CX_ERR_UNSUPPORTED


@pytest.mark.parametrize("N", [1280, 1024])
def test_split16_psf_matches_fp64_oracle(N):
    """The 4f PSF with its column transforms on the tensor cores (precision
    "split16") against the FP64 oracle, at the headline configuration's optics
    (f_obj 8 mm, f_tube 200 mm, NA 0.6, n 1.33, 3 wavelengths, 6.5 um camera
    pitch) on 3 defocus planes: relative L2 <= 1e-5, and within 3x of the
    plain FP32 path's own error."""
    import torch

    import chromatix_b200 as cx
    import chromatix_b200.functional as cf
    from oracle import chromatix_oracle as O
    from tests.helpers import rel

    wl = np.array([0.45, 0.532, 0.63])
    dxw = 200000.0 * wl / (1.33 * N * 6.5)
    dx = np.stack([dxw, dxw], -1)
    rng = np.random.default_rng(5)
    z = np.array([-4.0, 0.3, 5.0])
    phase = rng.uniform(0, 2 * np.pi, (N, N)).astype(np.float32)

    def run(prec):
        with cx.precision(prec):
            f = cf.objective_point_source((N, N), dx, (wl, np.ones(3)), z, 8000.0, 1.33, 0.6)
            f = cf.ff_lens(cf.phase_change(f, torch.as_tensor(phase, device="cuda")), 200000.0, 1.33)
            return f.intensity.cpu().numpy()

    I16, I32 = run("split16"), run("accurate")
    assert np.isfinite(I16).all()
    O.set_fft_workers(8)
    ref = O.ff_lens(O.phase_change(O.objective_point_source((N, N), dx, (wl, np.ones(3)), z, 8000.0, 1.33, 0.6),
                                   phase), 200000.0, 1.33).intensity
    e16, e32 = rel(I16, ref), rel(I32, ref)
    assert e16 < 1e-5, (e16, e32)
    assert e16 < 3 * e32 + 1e-6, (e16, e32)
