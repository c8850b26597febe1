"""Incoherent imaging on the GPU: fourier_convolution and the Microscope
(4f PSF -> plane-wise convolution -> sensor sum) against the FP64 oracle.
Tolerance: relative L2 <= 1e-5."""

import numpy as np
import pytest

from oracle import chromatix_oracle as O
from tests.helpers import rel, to_np

pytestmark = pytest.mark.gpu


# shapes cover power-of-two and 3/5/7-smooth transform lengths, odd half row
# lengths (w = 5, 7: M = 5, 7, no first-stage zero mask), single rows and
# columns
SHAPES = [(3, 40, 56), (2, 37, 29), (1, 64, 64), (4, 5, 2), (2, 96, 130), (2, 9, 7), (3, 6, 5), (2, 1, 1),
          (3, 1, 7), (2, 7, 1), (1, 100, 140), (2, 700, 300), (1, 190, 1800)]


@pytest.mark.parametrize("lengths", ["smallest", "pow2"])
@pytest.mark.parametrize("shape", SHAPES)
def test_fourier_convolution_matches_oracle(shape, lengths):
    import torch

    from chromatix_b200.ops import fourier_convolution

    rng = np.random.default_rng(sum(shape))
    a = rng.standard_normal(shape).astype(np.float32)
    k = rng.uniform(0, 1, shape).astype(np.float32)
    ad, kd = torch.as_tensor(a, device="cuda"), torch.as_tensor(k, device="cuda")
    ref = O.fourier_convolution(a.astype(np.float64), k.astype(np.float64), axes=(-2, -1))
    out = fourier_convolution(ad, kd, lengths=lengths)
    assert tuple(out.shape) == shape
    assert rel(to_np(out), ref) < 1e-5
    red = fourier_convolution(ad, kd, reduce=True, lengths=lengths)
    assert rel(to_np(red), ref.sum(0)) < 1e-5


def test_fourier_convolution_published_plane_size():
    """1536^2 planes (the reference's imaging benchmark): 3072-point
    transforms against the FP64 oracle's 4096-point ones, and the plane sum
    of 24 planes (more than one row-spectrum chunk) against the per-plane
    images summed in FP64."""
    import torch

    from chromatix_b200.ops import fourier_convolution

    rng = np.random.default_rng(1536)
    shape = (24, 1536, 1536)
    a = torch.rand(shape, device="cuda", generator=torch.Generator("cuda").manual_seed(1))
    k = torch.rand(shape, device="cuda", generator=torch.Generator("cuda").manual_seed(2))
    per = fourier_convolution(a, k)
    red = fourier_convolution(a, k, reduce=True)
    assert rel(to_np(red), to_np(per).astype(np.float64).sum(0)) < 1e-5
    for i in rng.choice(24, 2, replace=False):
        ref = O.fourier_convolution(to_np(a[i]).astype(np.float64), to_np(k[i]).astype(np.float64), axes=(-2, -1))
        assert rel(to_np(per[i]), ref) < 1e-5
    pow2 = fourier_convolution(a[:3], k[:3], reduce=True, lengths="pow2")
    assert rel(to_np(pow2), to_np(per[:3]).astype(np.float64).sum(0)) < 1e-5


@pytest.mark.parametrize("ha,hb,fast", [(512, 256, True), (513, 253, False)])
def test_fourier_convolution_reference_cases(ha, hb, fast):
    """The reference's own cases (tests/test_convolution.py:8-41): a kernel
    smaller than the image, scipy's "same" convolution, atol 1e-3 there; the
    FP64 oracle and relative L2 1e-5 here."""
    import torch

    from chromatix_b200.ops import fourier_convolution

    rng = np.random.default_rng(ha)
    a, b = rng.standard_normal((ha, ha)), rng.standard_normal((hb, hb))
    out = fourier_convolution(torch.as_tensor(a, dtype=torch.float32, device="cuda"),
                              torch.as_tensor(b, dtype=torch.float32, device="cuda"), fast_fft_shape=fast)
    ref = O.fourier_convolution(a, b, fast_fft_shape=fast)
    assert tuple(out.shape) == (ha, ha)
    assert np.allclose(to_np(out), ref, atol=1e-3)
    assert rel(to_np(out), ref) < 1e-5


@pytest.mark.parametrize("lengths", ["smallest", "pow2"])
@pytest.mark.parametrize("shape,kshape", [((3, 40, 56), (3, 9, 13)), ((2, 21, 17), (2, 40, 33)),
                                          ((4, 30, 31), (1, 7, 8)), ((2, 1, 9), (2, 5, 1))])
def test_fourier_convolution_unequal_kernels(shape, kshape, lengths):
    """Kernels smaller and larger than the image, per plane or one for all
    planes (broadcast), with and without the plane sum."""
    import torch

    from chromatix_b200.ops import fourier_convolution

    rng = np.random.default_rng(sum(shape) + sum(kshape))
    a = rng.standard_normal(shape).astype(np.float32)
    k = rng.uniform(-1, 1, kshape).astype(np.float32)
    kb = np.broadcast_to(k, shape[:1] + kshape[1:]).astype(np.float64)
    ref = np.stack([O.fourier_convolution(a[i].astype(np.float64), kb[i]) for i in range(shape[0])])
    ad, kd = torch.as_tensor(a, device="cuda"), torch.as_tensor(k, device="cuda")
    out = fourier_convolution(ad, kd, lengths=lengths)
    assert tuple(out.shape) == shape
    assert rel(to_np(out), ref) < 1e-5
    red = fourier_convolution(ad, kd, reduce=True, lengths=lengths)
    assert rel(to_np(red), ref.sum(0)) < 1e-5


def test_fourier_convolution_rejects_unsupported_forms():
    import torch

    from chromatix_b200.ops import fourier_convolution

    a = torch.zeros((2, 16, 16), device="cuda")
    with pytest.raises(NotImplementedError):
        fourier_convolution(a, torch.zeros((3, 8, 8), device="cuda"))
    with pytest.raises(AssertionError):
        fourier_convolution(a, torch.zeros((8, 8), device="cuda"))
    with pytest.raises(NotImplementedError):
        fourier_convolution(a, a, mode="full")
    with pytest.raises(NotImplementedError):
        fourier_convolution(a.to(torch.complex64), a.to(torch.complex64))
    with pytest.raises(ValueError):
        fourier_convolution(a, a, lengths="exact")
    big = torch.zeros((1, 2049, 8), device="cuda")
    with pytest.raises(Exception, match="longer than 4096"):
        fourier_convolution(big, big)


def test_microscope_image_matches_oracle():
    """systems/microscopes.py:271-297 with Optical4FSystemPSF and
    BasicSensor(resampling_method=None, reduce_axis=0), as in docs/parallelism.md."""
    import torch

    from chromatix_b200.systems import BasicSensor, Microscope, Optical4FSystemPSF

    shape, spacing, lam, f, n, NA, f_tube = (96, 96), 0.3, 0.532, 100.0, 1.33, 0.8, 200.0
    z = np.linspace(-4, 4, 5)
    rng = np.random.default_rng(3)
    phase = rng.uniform(0, 0.5, shape).astype(np.float32)
    sample = rng.uniform(0, 1, (5,) + shape).astype(np.float32)
    scope = Microscope(Optical4FSystemPSF(shape, spacing, f_tube, phase),
                       BasicSensor(shape, spacing, resampling_method=None, reduce_axis=0), f, n, NA, lam)
    img = scope(torch.as_tensor(sample, device="cuda"), z)
    ref, _ = O.microscope_image(sample.astype(np.float64), shape, spacing, f_tube, phase, f, n, NA, lam, z)
    assert tuple(img.shape) == shape
    assert rel(to_np(img), ref) < 1e-5
    # without a reduction: one image per plane
    scope2 = Microscope(Optical4FSystemPSF(shape, spacing, f_tube, phase),
                        BasicSensor(shape, spacing, resampling_method=None), f, n, NA, lam)
    per_plane = scope2(torch.as_tensor(sample, device="cuda"), z)
    assert tuple(per_plane.shape) == (5,) + shape
    assert rel(to_np(per_plane).sum(0), ref) < 1e-5
