"""The oracle's fourier_convolution (ops/ops.py:9-86) against scipy's
fftconvolve "same" (no GPU)."""

import numpy as np
from scipy.signal import fftconvolve

from oracle import chromatix_oracle as O


def test_fourier_convolution_matches_scipy_same():
    rng = np.random.default_rng(0)
    for shape in [(40, 56), (37, 29), (1, 8), (64, 64)]:
        a, k = rng.standard_normal(shape), rng.standard_normal(shape)
        assert O.rel_l2(O.fourier_convolution(a, k, axes=(0, 1)), fftconvolve(a, k, mode="same")) < 1e-12
    a, k = rng.standard_normal((3, 20, 24)), rng.standard_normal((3, 20, 24))
    c = O.fourier_convolution(a, k, axes=(-2, -1))
    ref = np.stack([fftconvolve(a[i], k[i], mode="same") for i in range(3)])
    assert O.rel_l2(c, ref) < 1e-12


def test_fourier_convolution_reference_cases():
    """The reference's own cases (tests/test_convolution.py:8-41): a 512^2
    image with a 256^2 kernel at power-of-two lengths and 513^2 with 253^2 at
    the summed lengths, against scipy's "same" convolution (atol 1e-3 there)."""
    rng = np.random.default_rng(1)
    for (ha, hb), fast in [((512, 256), True), ((513, 253), False)]:
        a, b = rng.standard_normal((ha, ha)), rng.standard_normal((hb, hb))
        c = O.fourier_convolution(a, b, fast_fft_shape=fast)
        ref = fftconvolve(a, b, mode="same")
        assert c.shape == a.shape
        assert np.allclose(c, ref, atol=1e-3) and O.rel_l2(c, ref) < 1e-12


def test_basic_sensor_reduce_and_next_order():
    x = np.arange(24.0).reshape(2, 3, 4)
    np.testing.assert_array_equal(O.basic_sensor_reduce(x, 0), x.sum(0))
    assert O.next_order(3072) == 4096 and O.next_order(4096) == 4096 and O.next_order(3) == 4


def test_microscope_reads_the_psf_intensity_once():
    """Microscope.__call__ (systems/microscopes.py:232-269) evaluates the PSF
    field's intensity -- the whole PSF pipeline -- exactly once per image."""
    import torch

    from chromatix_b200.systems import BasicSensor, Microscope

    class CountingField:
        reads = 0

        @property
        def intensity(self):
            CountingField.reads += 1
            return torch.ones((4, 8, 8))

    class HostMicroscope(Microscope):
        def image(self, sample, psf, key=None):  # the convolution itself runs on the GPU only
            return psf.sum(0)

    scope = HostMicroscope(lambda microscope, *a: CountingField(),
                           BasicSensor((8, 8), 0.3, resampling_method=None, reduce_axis=0), 100.0, 1.33, 0.8, 0.532)
    out = scope(torch.zeros((4, 8, 8)), np.linspace(-1, 1, 4))
    assert CountingField.reads == 1
    assert tuple(out.shape) == (8, 8)
    # the sensor reads a field's intensity once too
    CountingField.reads = 0
    assert tuple(BasicSensor((8, 8), 0.3, resampling_method=None, reduce_axis=0)(CountingField()).shape) == (8, 8)
    assert CountingField.reads == 1
