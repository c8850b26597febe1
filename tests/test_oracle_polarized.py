"""The oracle's birefringent multislice (functional/samples.py:444-546): the
reference has no test of it, so the restatement is pinned by exact
properties: one slice is affine in the potential (u(V) = P u + H V Q u), the
projector Q is transverse (k . (Q x) = 0 for propagating k), and a zero
potential with NA 0 blocks everything (no GPU)."""

import numpy as np

from oracle import chromatix_oracle as O


def _u(shape, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(shape + (3,)) + 1j * rng.standard_normal(shape + (3,))


def test_one_slice_is_affine_in_the_potential():
    u = _u((12, 10), 0)
    V = np.random.default_rng(1).uniform(-0.05, 0.05, (1, 12, 10, 3, 3))
    a = O.polarized_multislice_thick_sample(u, 0.3, 0.532, 0 * V, 1.33, 0.5)
    b = O.polarized_multislice_thick_sample(u, 0.3, 0.532, V, 1.33, 0.5)
    c = O.polarized_multislice_thick_sample(u, 0.3, 0.532, 2.5 * V, 1.33, 0.5)
    assert O.rel_l2(c - a, 2.5 * (b - a)) < 1e-12
    assert O.rel_l2(b, a) > 1e-4


def test_zero_na_blocks_the_field():
    u = _u((8, 8), 2)
    out = O.polarized_multislice_thick_sample(u, 0.3, 0.532, np.zeros((2, 8, 8, 3, 3)), 1.0, 0.5, NA=0.0)
    # only the DC column passes an NA of 0 (|k_perp| = 0 <= 0): a constant field
    np.testing.assert_allclose(out, np.broadcast_to(out[:1, :1], out.shape), atol=1e-12)


def test_projector_is_transverse():
    km = 2 * np.pi * 1.33 / 0.532
    rng = np.random.default_rng(3)
    for _ in range(20):
        kp = rng.uniform(-0.9, 0.9, 2) * km / np.sqrt(2)
        k = np.array([np.sqrt(km**2 - kp @ kp), *kp]) / km
        Q = np.eye(3) - np.outer(k, k)
        x = rng.standard_normal(3) + 1j * rng.standard_normal(3)
        assert abs(k @ (Q @ x)) < 1e-12
