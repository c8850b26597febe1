"""The oracle's fluorescent thick sample (functional/samples.py:285-441) pinned
by known answers (the reference has no test of it): with every frequency
propagating, the forward and backward slice kernels cancel, so the stack
reproduces the field propagated to each slice plane; a lone fluorescent slice
comes back as its own intensity; the phase generator is deterministic and
uniform on [0, 2 pi) (no GPU)."""

import numpy as np

from oracle import chromatix_oracle as O


def _field(shape, dx, lam, seed):
    rng = np.random.default_rng(seed)
    u = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    return O.field_build(u, dx, lam)


def test_one_slice_without_fluorescence_returns_the_input_intensity():
    # dx = 1 um, lambda = 0.5 um: lambda f <= 0.25, every frequency propagates
    f = _field((24, 20), 1.0, 0.5, 0)
    dn = np.random.default_rng(1).uniform(-0.05, 0.05, (1, 24, 20))
    I = O.fluorescent_multislice_thick_sample(f, np.zeros_like(dn), dn, 1.33, 0.7, 6, np.zeros((1, 1, 24, 20)))
    np.testing.assert_allclose(I[0], np.abs(f.u) ** 2, rtol=1e-9, atol=1e-12)


def test_stack_is_the_field_propagated_to_each_slice_plane():
    f = _field((16, 16), 1.0, 0.5, 2)
    D, dz, n, pad = 4, 2.0, 1.0, 8
    z = np.zeros((D, 16, 16))
    I = O.fluorescent_multislice_thick_sample(f, z, z, n, dz, pad, np.zeros((1, D, 16, 16)))
    for j in range(D):
        # I[j]: the padded input propagated by j slices (asm_propagate returns the padded grid)
        pj = O.crop(O.asm_propagate(f, j * dz, n, pad), pad) if j else f
        np.testing.assert_allclose(I[j], np.abs(pj.u) ** 2, rtol=1e-8, atol=1e-10)


def test_lone_fluorescent_slice_returns_its_intensity():
    f = O.field_build(np.zeros((20, 20), complex), 1.0, 0.5)
    fl = np.zeros((1, 20, 20))
    fl[0] = np.random.default_rng(3).uniform(0, 1, (20, 20))
    ph = np.random.default_rng(4).uniform(0, 2 * np.pi, (1, 1, 20, 20))
    I = O.fluorescent_multislice_thick_sample(f, fl, np.zeros_like(fl), 1.2, 1.5, 4, ph)
    np.testing.assert_allclose(I[0], fl[0] ** 2, rtol=1e-9, atol=1e-12)


def test_phase_generator():
    a = O.fluor_phases(7, 0, (3, 16, 16))
    b = O.fluor_phases(7, 0, (3, 16, 16))
    c = O.fluor_phases(7, 1, (3, 16, 16))
    np.testing.assert_array_equal(a, b)
    assert a.dtype == np.float32 and not np.array_equal(a, c)
    x = O.fluor_phases(11, 0, (1 << 16,))
    assert x.min() >= 0 and x.max() < 2 * np.pi
    assert abs(x.mean() - np.pi) < 0.03 and abs(x.std() - 2 * np.pi / np.sqrt(12)) < 0.02
