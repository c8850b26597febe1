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


def test_basic_sensor_reduce_and_next_order():
    x = np.arange(24.0).reshape(2, 3, 4)
    np.testing.assert_array_equal(O.basic_sensor_reduce(x, 0), x.sum(0))
    assert O.next_order(3072) == 4096 and O.next_order(4096) == 4096 and O.next_order(3) == 4
