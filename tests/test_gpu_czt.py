"""Chirp-Z transforms and the rescaled (CZT) propagation on the GPU vs the
oracle / numpy / scipy (relative L2 <= 1e-5 unless stated)."""

import numpy as np
import pytest
from scipy.signal import czt as czt_scipy

from oracle import chromatix_oracle as O
from tests.helpers import cuda_field, oracle_field, rand_field, rel, to_np

pytestmark = pytest.mark.gpu


def _x(shape, seed=42):
    rng = np.random.default_rng(seed)
    return (rng.uniform(size=shape) + 1j * rng.uniform(size=shape)).astype(np.complex64)


def test_czt_as_dft_and_idft():
    """tests/test_czt.py:15-40 on the CUDA path."""
    import torch

    from chromatix_b200.utils import czt

    N = M = 100
    x = _x((N, N))
    xt = torch.as_tensor(x, device="cuda")
    w = np.exp(-1j * 2 * np.pi / N)
    for axis in range(2):
        assert rel(to_np(czt(xt, M, 1.0, w, axis=axis)), np.fft.fft(x.astype(np.complex128), axis=axis)) < 1e-5
    w = np.exp(1j * 2 * np.pi / N)
    for axis in range(2):
        assert rel(to_np(czt(xt, M, 1.0, w, axis=axis)) / N, np.fft.ifft(x.astype(np.complex128), axis=axis)) < 1e-5


def test_czt_against_scipy_and_general_a_w():
    import torch

    from chromatix_b200.utils import czt

    rng = np.random.default_rng(0)
    # the last two need Bluestein lengths above 4096 (4608 and 6144)
    for (n, m) in [(100, 10), (37, 211), (1024, 512), (5, 3), (4096, 512), (3000, 3000)]:
        x = (rng.standard_normal((7, n)) + 1j * rng.standard_normal((7, n))).astype(np.complex64)
        a = np.exp(1j * 0.3)
        w = np.exp(-1j * 2 * np.pi / (1.7 * n))
        ref = czt_scipy(x.astype(np.complex128), a=a, w=w, m=m, axis=-1)
        out = to_np(czt(torch.as_tensor(x, device="cuda"), m, a, w, axis=-1))
        assert rel(out, ref) < 1e-5, (n, m)
        # strided axis (column tiles)
        out0 = to_np(czt(torch.as_tensor(np.ascontiguousarray(x.T), device="cuda"), m, a, w, axis=0))
        assert rel(out0, ref.T) < 1e-5, (n, m)


def test_cztn_and_zoomed_fft():
    import torch

    from chromatix_b200.utils import cztn, zoomed_fft

    x = _x((3, 64, 48), seed=1)
    xt = torch.as_tensor(x, device="cuda")
    N = 64
    w = np.exp(-1j * 2 * np.pi / N)
    ref = O.cztn(x.astype(np.complex128), (40, 30), (1, 1), (w, np.exp(-1j * 2 * np.pi / 48)), axes=(1, 2))
    out = to_np(cztn(xt, (40, 30), (1, 1), (w, np.exp(-1j * 2 * np.pi / 48)), axes=(1, 2)))
    assert rel(out, ref) < 1e-5
    refz = O.zoomed_fft(x.astype(np.complex128), -0.3 * np.pi, 0.3 * np.pi, (33, 65), axes=(1, 2))
    outz = to_np(zoomed_fft(xt, -0.3 * np.pi, 0.3 * np.pi, (33, 65), axes=(1, 2)))
    assert rel(outz, refz) < 1e-5


@pytest.mark.parametrize("fn", ["asm_propagate", "transfer_propagate"])
@pytest.mark.parametrize("zoom,shape_out,pad", [(2.0, (128, 96), 64), (0.5, (64, 64), 32), (1.3, (100, 120), 0)])
def test_rescaled_czt_propagation(fn, zoom, shape_out, pad):
    import chromatix_b200.functional as cf

    u = rand_field((128, 128), seed=2)
    dx = 0.3
    kw = dict(output_dx=np.array([dx / zoom, dx / zoom]), output_shape=shape_out)
    out = getattr(cf, fn)(cuda_field(u, dx, 0.532), 40.0, 1.33, pad, **kw)
    ref = getattr(O, fn)(oracle_field(u, dx, 0.532), 40.0, 1.33, pad, **kw)
    assert out.u.shape == ref.u.shape
    assert rel(to_np(out.u), ref.u) < 1e-5
    np.testing.assert_allclose(out.dx, ref.dx)


def test_rescaled_with_shift_and_same_mode():
    import chromatix_b200.functional as cf

    u = rand_field((128, 128), seed=3)
    kw = dict(output_dx=np.array([0.15, 0.15]), output_shape=(160, 160), shift_yx=(2.0, -3.0), mode="same")
    out = cf.asm_propagate(cuda_field(u, 0.3, 0.532), 25.0, 1.33, 16, **kw)
    ref = O.asm_propagate(oracle_field(u, 0.3, 0.532), 25.0, 1.33, 16, **kw)
    assert out.u.shape == ref.u.shape
    assert rel(to_np(out.u), ref.u) < 1e-5


@pytest.mark.parametrize("fn", ["asm_propagate", "transfer_propagate"])
@pytest.mark.parametrize("zoom,pad,shift,mode", [(2.0, 64, (0.0, 0.0), "full"), (0.5, 32, (1.5, -2.0), "full"),
                                                 (1.3, 0, (0.0, 0.0), "same"), (4.0, 48, (0.0, 0.0), "same")])
def test_rescaled_yu_branch(fn, zoom, pad, shift, mode):
    """kernel_propagate's use_czt=False branch (functional/propagation.py:445-458): the
    chirp convolution against the FP64 oracle (scipy fftconvolve)."""
    import chromatix_b200.functional as cf

    u = rand_field((128, 96), seed=4)
    dx = 0.3
    kw = dict(output_dx=np.array([dx / zoom, dx / zoom]), use_czt=False, shift_yx=shift, mode=mode)
    out = getattr(cf, fn)(cuda_field(u, dx, 0.532), 40.0, 1.33, pad, **kw)
    ref = getattr(O, fn)(oracle_field(u, dx, 0.532), 40.0, 1.33, pad, **kw)
    assert out.u.shape == ref.u.shape
    assert rel(to_np(out.u), ref.u) < 1e-5
    np.testing.assert_allclose(out.dx, ref.dx)


def test_rescaled_yu_branch_rejects_other_output_shapes():
    import chromatix_b200.functional as cf
    from chromatix_b200._native import CxError

    u = rand_field((64, 64), seed=5)
    with pytest.raises(CxError):
        cf.asm_propagate(cuda_field(u, 0.3, 0.532), 40.0, 1.33, 16, output_dx=np.array([0.15, 0.15]),
                         output_shape=(64, 64), use_czt=False)


@pytest.mark.parametrize("use_czt", [True, False])
def test_rescaled_band_limited(use_czt):
    """The band-limited (Matsushima) ASM propagator in both rescaled branches, as in
    docs/examples/rescaled_propagation.ipynb."""
    import chromatix_b200.functional as cf

    u = rand_field((128, 128), seed=6)
    kw = dict(output_dx=np.array([0.3 / 1.5] * 2), shift_yx=(3.0, -1.0), bandlimit=True, use_czt=use_czt,
              mode="same")
    out = cf.asm_propagate(cuda_field(u, 0.3, 0.532), 300.0, 1.0, 64, **kw)
    ref = O.asm_propagate(oracle_field(u, 0.3, 0.532), 300.0, 1.0, 64, **kw)
    assert out.u.shape == ref.u.shape
    assert rel(to_np(out.u), ref.u) < 1e-5
