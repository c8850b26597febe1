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
