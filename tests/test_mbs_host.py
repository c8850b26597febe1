"""Host-side pieces of the MBS module (no GPU): absorbing boundaries and the
shift/scale search on CPU tensors vs the oracle."""

import numpy as np


def test_absorbing_bc_matches_oracle():
    import torch

    from chromatix_b200.experimental import mbs
    from oracle import chromatix_oracle as O

    rng = np.random.default_rng(0)
    perm = (1 + 0.2 * rng.uniform(size=(6, 7, 5)) + 0.01j * rng.uniform(size=(6, 7, 5)))
    s = mbs.Sample(torch.as_tensor(perm.astype(np.complex64)), 0.1)
    for axis in (0, (0, 2), (0, 1, 2)):
        out = mbs.add_absorbing_bc(s, axis, 0.3, 0.25, 1.33)
        ref, roi = O.mbs_add_absorbing_bc(perm, 0.1, axis, 0.3, 0.25, 1.33)
        assert out.ROI == roi
        np.testing.assert_allclose(out.permittivity.numpy(), ref, rtol=1e-6, atol=1e-6)


def test_shift_and_scale_matches_exact_circle():
    import torch

    from chromatix_b200.experimental import mbs
    from oracle import chromatix_oracle as O

    rng = np.random.default_rng(1)
    perm = (1.2 + 0.3 * rng.standard_normal((10, 10, 10)) + 0.05j * rng.uniform(size=(10, 10, 10))) ** 2
    c0, s0 = O.mbs_shift_and_scale(perm)
    c, s = mbs.get_shift_and_scale(torch.as_tensor(perm.astype(np.complex64)), n_directions=256)
    R0, R = abs(1 / s0), abs(1 / s)
    # the scale always covers every value (convergence of the series) ...
    assert R >= R0 * (1 - 1e-6)
    # ... and is within a fraction of a percent of the optimum
    assert R <= R0 * 1.005
    assert abs(c - c0) < 0.01 * R0
