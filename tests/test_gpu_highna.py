"""high_na_ff_lens (functional/lenses.py:98-156) on the GPU against the FP64
oracle: scalar and vector fields (the spherical basis change of
core/field.py:897-940), non-square and odd output grids, a pupil grid that
reaches the evanescent region (sz = 0: zero defocus weight), batched fields,
a shifted origin.  Tolerance: relative L2 <= 1e-5."""

import numpy as np
import pytest

from oracle import chromatix_oracle as O
from tests.helpers import rel, to_np

pytestmark = pytest.mark.gpu

CASES = [
    # shape, dx, lam, f, n, NA, output_shape, output_dx
    ((64, 64), 0.5, 0.532, 100.0, 1.33, 0.8, None, None),
    ((64, 64), 0.5, 0.532, 100.0, 1.33, 0.8, (48, 56), 0.3),
    ((45, 45), 0.4, 0.6, 250.0, 1.0, 0.5, (31, 33), 0.7),
    ((96, 96), 0.2, 0.532, 60.0, 1.0, 0.95, (80, 80), 0.25),  # NA lambda / (2 n dx) > 1: evanescent corner
]


def _rand(shape, seed):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)


@pytest.mark.parametrize("case", range(len(CASES)))
@pytest.mark.parametrize("vectorial", [False, True])
def test_high_na_ff_lens_matches_oracle(case, vectorial):
    import torch

    import chromatix_b200 as cx
    import chromatix_b200.functional as cf

    shape, dx, lam, f, n, NA, oshape, odx = CASES[case]
    u = _rand(shape + ((3,) if vectorial else ()), 10 * case + vectorial)
    field = cx.Field.build(torch.as_tensor(u, device="cuda"), dx, lam)
    assert isinstance(field, cx.VectorField) == vectorial
    out = cf.high_na_ff_lens(field, f, n, NA, output_shape=oshape, output_dx=odx)
    ref, rdx = O.high_na_ff_lens(u.astype(np.complex128), dx, lam, f, n, NA, output_shape=oshape, output_dx=odx)
    assert tuple(out.u.shape) == ref.shape
    assert rel(to_np(out.u), ref) < 1e-5
    np.testing.assert_allclose(out.dx, rdx)


def test_high_na_ff_lens_batched_fields_and_shifted_origin():
    import torch

    import chromatix_b200 as cx
    import chromatix_b200.functional as cf

    u = _rand((3, 40, 40, 3), 7)
    field = cx.shift_grid(cx.VectorField(torch.as_tensor(u, device="cuda"), 0.3, 0.0, cx.MonoSpectrum(0.5)),
                          (0.45, -0.6))
    out = cf.high_na_ff_lens(field, 20.0, 1.0, 0.9, output_shape=(36, 30), output_dx=0.1)
    for b in range(3):
        ref, _ = O.high_na_ff_lens(u[b].astype(np.complex128), 0.3, 0.5, 20.0, 1.0, 0.9, output_shape=(36, 30),
                                   output_dx=0.1, origin=(0.45, -0.6))
        assert rel(to_np(out.u[b]), ref) < 1e-5
    # the vector intensity sums the components
    I = to_np(out.intensity)
    np.testing.assert_allclose(I, np.sum(np.abs(to_np(out.u)) ** 2, -1), rtol=1e-5)


def test_high_na_ff_lens_rejects_unsupported_forms():
    import torch

    import chromatix_b200 as cx
    import chromatix_b200.functional as cf
    from chromatix_b200._native import CxError

    field = cx.Field.build(torch.zeros((16, 16), dtype=torch.complex64, device="cuda"), 0.5, 0.5)
    with pytest.raises(CxError):
        cf.high_na_ff_lens(field, 10.0, 1.0, 0.5, output_shape=(1, 8))
    chrom = cx.Field.build(torch.zeros((16, 16, 2), dtype=torch.complex64, device="cuda"), 0.5,
                           (np.array([0.5, 0.6]), np.ones(2)))
    with pytest.raises(NotImplementedError):
        cf.high_na_ff_lens(chrom, 10.0, 1.0, 0.5)
