"""polarized_multislice_thick_sample (functional/samples.py:444-546) on the
GPU against the FP64 oracle: square and non-square grids, NA 1 and below,
a grid reaching the evanescent region (kz = 0: no free-space or scattering
transfer there).  Tolerance: relative L2 <= 1e-5.

With NA = 1 the wavelengths are chosen so that no frequency of the padded
grid lies on the circle |k_perp| = km (n / lambda = 2.5 puts the padded
grid's Nyquist row there for dx = 0.2): on that circle kz is zero up to
rounding and the scattering factor dz / (2 kz) takes whatever value the
rounding gives, in the reference as in any restatement."""

import numpy as np
import pytest

from oracle import chromatix_oracle as O
from tests.helpers import rel, to_np

pytestmark = pytest.mark.gpu

CASES = [
    # shape, D, dx, NA, dz, lambda
    ((32, 24), 3, 0.2, 1.0, 0.5, 0.55),
    ((16, 16), 5, 0.3, 0.6, 0.8, 0.532),
    ((40, 56), 2, 0.25, 0.9, 1.0, 0.532),
    ((64, 64), 4, 0.1, 1.0, 0.3, 0.55),  # dx < lambda / (2 n): evanescent corners
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_polarized_multislice_matches_oracle(case):
    import torch

    import chromatix_b200 as cx
    import chromatix_b200.functional as cf

    shape, D, dx, NA, dz, lam = CASES[case]
    rng = np.random.default_rng(case)
    u = (rng.standard_normal(shape + (3,)) + 1j * rng.standard_normal(shape + (3,))).astype(np.complex64)
    V = rng.uniform(-0.05, 0.05, (D,) + shape + (3, 3)).astype(np.float32)
    f = cx.Field.build(torch.as_tensor(u, device="cuda"), dx, lam)
    out = cf.polarized_multislice_thick_sample(f, torch.as_tensor(V, device="cuda"), 1.33, dz, NA)
    ref = O.polarized_multislice_thick_sample(u.astype(np.complex128), dx, lam, V.astype(np.float64), 1.33, dz, NA)
    assert tuple(out.u.shape) == ref.shape
    assert rel(to_np(out.u), ref) < 1e-5


def test_polarized_multislice_rejects_unsupported_forms():
    import torch

    import chromatix_b200 as cx
    import chromatix_b200.functional as cf
    from chromatix_b200._native import CxError

    odd = cx.Field.build(torch.zeros((15, 16, 3), dtype=torch.complex64, device="cuda"), 0.2, 0.5)
    with pytest.raises(CxError, match="even field sizes"):
        cf.polarized_multislice_thick_sample(odd, np.zeros((1, 15, 16, 3, 3), np.float32), 1.0, 0.5)
    scalar = cx.Field.build(torch.zeros((16, 16), dtype=torch.complex64, device="cuda"), 0.2, 0.5)
    with pytest.raises(AssertionError):
        cf.polarized_multislice_thick_sample(scalar, np.zeros((1, 16, 16, 3, 3), np.float32), 1.0, 0.5)


def test_polarized_multislice_chromatic_vector_field():
    """A ChromaticVectorField: every wavelength through the same potential
    (the reference broadcasts it over the wavelength axis), with its own
    spacing and wavenumber."""
    import torch

    import chromatix_b200 as cx
    import chromatix_b200.functional as cf

    wl = np.array([0.47, 0.55, 0.61])
    rng = np.random.default_rng(9)
    u = (rng.standard_normal((24, 32, 3, 3)) + 1j * rng.standard_normal((24, 32, 3, 3))).astype(np.complex64)
    V = rng.uniform(-0.05, 0.05, (3, 24, 32, 3, 3)).astype(np.float32)
    f = cx.Field.build(torch.as_tensor(u, device="cuda"), 0.2, (wl, np.ones(3)))
    assert isinstance(f, cx.ChromaticVectorField)
    out = to_np(cf.polarized_multislice_thick_sample(f, torch.as_tensor(V, device="cuda"), 1.33, 0.5, 1.0).u)
    for w in range(3):
        ref = O.polarized_multislice_thick_sample(u[:, :, w].astype(np.complex128), 0.2, wl[w],
                                                  V.astype(np.float64), 1.33, 0.5, 1.0)
        assert rel(out[:, :, w], ref) < 1e-5
