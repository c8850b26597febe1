"""The FFT engine on the GPU vs numpy, for every compiled length (cx_fft1d)."""

import numpy as np
import pytest

from tests.helpers import to_np

SIZES = [2, 3, 4, 5, 6, 7, 8, 10, 12, 14, 16, 20, 24, 28, 32, 40, 48, 56, 64, 80, 96, 112, 128, 160, 192, 224, 256,
         320, 384, 448, 512, 640, 768, 896, 1024, 1280, 1536, 1792, 2048, 2560, 3072, 3584, 4096,
         4608, 5120, 6144, 7168, 8192]  # the last five: 1D / chirp-Z lengths only


@pytest.mark.gpu
@pytest.mark.parametrize("n", SIZES)
def test_fft1d_matches_numpy(n):
    import torch

    from chromatix_b200 import _native as nat

    rng = np.random.default_rng(n)
    batch = 37
    x = (rng.standard_normal((batch, n)) + 1j * rng.standard_normal((batch, n))).astype(np.complex64)
    xd = torch.as_tensor(x, device="cuda")
    y = torch.empty_like(xd)
    L = nat.lib()
    for inv in (0, 1):
        nat.check(L.cx_fft1d(nat.ptr(xd), nat.ptr(y), n, batch, inv, nat.stream_handle()))
        torch.cuda.synchronize()
        ref = np.fft.ifft(x.astype(np.complex128), axis=-1) if inv else np.fft.fft(x.astype(np.complex128), axis=-1)
        err = np.linalg.norm(to_np(y) - ref) / np.linalg.norm(ref)
        assert err < 2e-6, (n, inv, err)


@pytest.mark.gpu
def test_fft1d_unsupported_length_is_an_error():
    import torch

    from chromatix_b200 import _native as nat

    x = torch.zeros(11 * 13, dtype=torch.complex64, device="cuda")
    with pytest.raises(nat.CxError):
        nat.check(nat.lib().cx_fft1d(nat.ptr(x), nat.ptr(x), 143, 1, 0, nat.stream_handle()))


@pytest.mark.gpu
def test_fft1d_empty_batch_is_a_no_op():
    import torch

    from chromatix_b200 import _native as nat

    x = torch.zeros(8, dtype=torch.complex64, device="cuda")
    y = torch.full_like(x, 3.0)
    nat.check(nat.lib().cx_fft1d(nat.ptr(x), nat.ptr(y), 8, 0, 0, nat.stream_handle()))
    torch.cuda.synchronize()
    assert torch.all(y == 3.0)
