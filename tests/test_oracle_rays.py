"""The oracle's ray transfer (functional/rays.py:102-154) pinned by known
answers (the reference has no test of it): free space with unit
magnification is the Fresnel transfer-function propagation; a Gaussian beam
through a lens and a focal length of free space focuses to the paraxial
waist lambda f / (pi w0); every ABCD system conserves the field's summed
intensity; the ABCD products follow the reference's matrices (no GPU)."""

import numpy as np

from oracle import chromatix_oracle as O


def _field(shape, dx, lam, seed):
    rng = np.random.default_rng(seed)
    return O.field_build(rng.standard_normal(shape) + 1j * rng.standard_normal(shape), dx, lam)


def test_free_space_is_transfer_propagation():
    f = _field((32, 28), 0.5, 0.532, 0)
    out = O.ray_transfer(f, [[1.0, 40.0], [0.0, 1.0]], 1.33)
    ref = O.transfer_propagate(f, 40.0, 1.33, 0)
    assert O.rel_l2(out.u, ref.u) < 1e-12
    np.testing.assert_allclose(out.dx, f.dx)


def test_summed_intensity_is_conserved():
    f = _field((24, 24), 0.4, 0.6, 1)
    lens = np.array([[1.0, 0.0], [-1 / 50.0, 1.0]])
    free = np.array([[1.0, 30.0], [0.0, 1.0]])
    for abcd, m in [(free @ lens, 1.0), (free @ lens, 1.7), (np.array([[0.3, 12.0], [-0.05, 1.4]]), 0.6)]:
        out = O.ray_transfer(f, abcd, 1.0, m)
        np.testing.assert_allclose(np.sum(np.abs(out.u) ** 2), np.sum(np.abs(f.u) ** 2), rtol=1e-12)
        np.testing.assert_allclose(out.dx, f.dx / m)


def test_abcd_matrices():
    from chromatix_b200.functional import rays as R

    np.testing.assert_array_equal(R.compute_free_space_abcd(3.0), [[1, 3], [0, 1]])
    np.testing.assert_array_equal(R.compute_thin_spherical_lens_abcd(4.0, inverse=True), [[1, 0], [0.25, 1]])
    # a thick plano-convex lens of zero thickness acts as a thin lens of power (n_l - n_m) / (R n_m)
    M = R.compute_plano_convex_spherical_lens_abcd(100.0, 50.0, 0.0, 1.5, 1.0)
    np.testing.assert_allclose(M, [[1, 0], [-0.5 / 50.0, 1]], atol=1e-15)


def test_gaussian_beam_focuses_to_its_paraxial_waist():
    # lambda B / M = 50 um <= N dx^2 = 64 um: the transfer function is sampled without aliasing
    N, dx, lam, f, w0 = 256, 0.5, 0.5, 100.0, 10.0
    g = (np.arange(N) - N / 2) * dx
    Y, X = np.meshgrid(g, g, indexing="ij")
    field = O.field_build(np.exp(-(X**2 + Y**2) / w0**2), dx, lam)
    lens = np.array([[1.0, 0.0], [-1 / f, 1.0]])
    free = np.array([[1.0, f], [0.0, 1.0]])
    out = O.ray_transfer(field, free @ lens, 1.0)
    I = np.abs(out.u) ** 2
    w = 2 * np.sqrt((I * X**2).sum() / I.sum())  # I ~ exp(-2 r^2 / w^2): <x^2> = w^2 / 4
    assert abs(w - lam * f / (np.pi * w0)) < 1e-3 * w
    np.testing.assert_allclose(I.sum(), (np.abs(field.u) ** 2).sum(), rtol=1e-12)
