"""Padding rules and argument validation of the propagation API (no GPU).

compute_padding_transform / _transfer / _exact follow the reference's Fresnel-
number rule (functional/propagation.py:583-656):
    Nf = (D/2)^2 / (lambda z), D = height dx,  Q = 2 max(1, M / (4 Nf)),
    exact: Q /= sqrt(1 - (lambda / (2 dx))^2),  N = 2 ceil(Q M / 2),  pad = N - M.
The expected values below are worked out by hand from that rule."""

import math

import numpy as np
import pytest

import chromatix_b200.functional as cf
from chromatix_b200.functional import propagation as P


def _rule(height, wavelength, dx, z, exact=False):
    D = height * dx
    Nf = (D / 2) ** 2 / (wavelength * z)
    Q = 2 * max(1.0, height / (4 * Nf))
    if exact:
        Q = Q / math.sqrt(1 - (wavelength / (2 * dx)) ** 2)
    return int(math.ceil(Q * height / 2) * 2) - height


@pytest.mark.parametrize("height,wl,dx,z,expect", [
    # Nf = (512*0.3/2)^2 / (0.532*100) = 110.87; M / (4 Nf) = 1.1545 -> Q = 2.309, N = 2 ceil(591.1) = 1184
    (512, 0.532, 0.3, 100.0, 672),
    # large Fresnel number: Q = 2 -> pad = M
    (256, 0.5, 1.0, 10.0, 256),
    # long distance: Nf = (64*0.5/2)^2 / (0.6*1e4) = 0.04267, M/(4Nf) = 375 -> N = 2 ceil(375*64) = 48000
    (64, 0.6, 0.5, 1e4, 47936),
])
def test_compute_padding_transform_and_transfer(height, wl, dx, z, expect):
    assert _rule(height, wl, dx, z) == expect
    assert cf.compute_padding_transform(height, wl, dx, z) == expect
    assert cf.compute_padding_transfer(height, wl, dx, z) == expect


@pytest.mark.parametrize("height,wl,dx,z", [(512, 0.532, 0.3, 100.0), (256, 0.5, 1.0, 10.0), (128, 0.5, 0.3, 50.0)])
def test_compute_padding_exact(height, wl, dx, z):
    got = cf.compute_padding_exact(height, wl, dx, z)
    assert got == _rule(height, wl, dx, z, exact=True)
    # the evanescent scale only ever enlarges the padding of the transfer rule
    assert got >= cf.compute_padding_transfer(height, wl, dx, z)


def test_compute_padding_exact_scale_case():
    # 512 px, dx = 0.3, lambda = 0.532: scale = 0.8867, Q = 2.309 / sqrt(1 - 0.7862) = 4.9935, N = 2 ceil(1278.3) = 2558
    Q = 2 * max(1.0, 512 / (4 * (512 * 0.3 / 2) ** 2 / (0.532 * 100.0)))
    Q /= math.sqrt(1 - (0.532 / 0.6) ** 2)
    assert cf.compute_padding_exact(512, 0.532, 0.3, 100.0) == int(math.ceil(Q * 256) * 2) - 512 == 2046


def test_absorbing_boundary_names_are_validated_before_any_device_work():
    # the reference asserts the name first (functional/propagation.py:382-385)
    with pytest.raises(AssertionError):
        P._check_boundary("gaussian")
    P._check_boundary(None)
    P._check_boundary("tukey")
    P._check_boundary("super_gaussian")
    with pytest.raises(AssertionError):
        cf.asm_propagate(object(), 1.0, 1.33, 0, absorbing_boundary="hann")
    with pytest.raises(AssertionError):
        cf.transfer_propagate(object(), 1.0, 1.33, 0, absorbing_boundary="hann")
    with pytest.raises(AssertionError):
        cf.kernel_propagate(object(), np.ones((4, 4)), absorbing_boundary="hann")
