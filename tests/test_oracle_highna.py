"""The oracle's high-NA lens (functional/lenses.py:98-156, core/field.py:
897-940) pinned by properties (the reference has no test of it): the
spherical basis change is a real orthogonal map of (Ex, Ey) per pupil pixel,
identity outside the pupil, and the zoomed FFT equals the explicit DFT at the
zoomed frequencies (no GPU)."""

import numpy as np

from oracle import chromatix_oracle as O


def test_spherical_basis_preserves_energy_and_is_identity_outside_the_pupil():
    rng = np.random.default_rng(0)
    shape, dx, f, n, NA = (32, 32), 0.4, 6.0, 1.33, 1.2
    u = rng.standard_normal(shape + (3,)) + 1j * rng.standard_normal(shape + (3,))
    g = O.pupil_grid(shape, dx)
    e = O.cartesian_to_spherical(u, g, n, NA, f)
    # per pixel |e|^2 = |Ex|^2 + |Ey|^2 (the z input component is not used)
    np.testing.assert_allclose(np.sum(np.abs(e) ** 2, -1), np.abs(u[..., 1]) ** 2 + np.abs(u[..., 2]) ** 2,
                               rtol=1e-12)
    outside = np.sum(g**2, -1) > (f * NA / n) ** 2
    assert outside.any() and (~outside).any()
    np.testing.assert_allclose(e[outside][:, 1:], u[outside][:, 1:], rtol=0, atol=1e-15)
    assert np.all(e[outside][:, 0] == 0)
    # on the axis (grid point (16, 16) = (0, 0)): the identity
    np.testing.assert_allclose(e[16, 16], [0, u[16, 16, 1], u[16, 16, 2]], rtol=0, atol=1e-15)


def test_zoomed_fft_equals_explicit_dft():
    rng = np.random.default_rng(1)
    x = rng.standard_normal((12, 10)) + 1j * rng.standard_normal((12, 10))
    k0, k1, m = -0.7 * np.pi, 0.9 * np.pi, (9, 7)
    z = O.zoomed_fft(x, k0, k1, m, axes=(0, 1), include_end=True)
    wy = k0 + (k1 - k0) * np.arange(m[0]) / (m[0] - 1)
    wx = k0 + (k1 - k0) * np.arange(m[1]) / (m[1] - 1)
    # y[k] = sum_j x[j] a^-j w^(jk) with a = exp(-i k0), w = exp(i dk): exp(+i omega_k j)
    Ey = np.exp(1j * np.outer(wy, np.arange(12)))
    Ex = np.exp(1j * np.outer(wx, np.arange(10)))
    np.testing.assert_allclose(z, Ey @ x @ Ex.T, rtol=0, atol=1e-10)


def test_high_na_lens_scalar_and_vector_agree_for_linear_polarisation_on_axis():
    """A scalar field equals the y component of the vector field Ey = u
    wherever the basis change is the identity: NA small enough that the pupil
    holds only the on-axis pixel's neighbourhood with cos(theta) ~ 1."""
    rng = np.random.default_rng(2)
    shape, dx, lam, f, n, NA = (24, 24), 0.5, 0.5, 1e6, 1.0, 0.3
    u = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    out_s, odx = O.high_na_ff_lens(u, dx, lam, f, n, NA, output_shape=(16, 16), output_dx=0.2)
    v = np.zeros(shape + (3,), complex)
    v[..., 1] = u
    out_v, _ = O.high_na_ff_lens(v, dx, lam, f, n, NA, output_shape=(16, 16), output_dx=0.2)
    assert odx == 0.2 and out_s.shape == (16, 16) and out_v.shape == (16, 16, 3)
    # f >> extent: sin(theta) ~ 1e-5, the basis change is the identity to ~1e-10
    assert O.rel_l2(out_v[..., 1], out_s) < 1e-8
    assert np.abs(out_v[..., 0]).max() < 1e-4 * np.abs(out_s).max()
