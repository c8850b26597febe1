"""ray_transfer (functional/rays.py:102-154) on the GPU against the FP64
oracle: free space (= transfer propagation), lens + free space, a general
ABCD with magnification, a chromatic batched field with a shifted origin.
Tolerance: relative L2 <= 1e-5."""

import numpy as np
import pytest

from oracle import chromatix_oracle as O
from tests.helpers import rel, to_np

pytestmark = pytest.mark.gpu

LENS = np.array([[1.0, 0.0], [-1 / 50.0, 1.0]])
FREE = np.array([[1.0, 30.0], [0.0, 1.0]])


@pytest.mark.parametrize("abcd,m", [(np.array([[1.0, 40.0], [0.0, 1.0]]), 1.0), (FREE @ LENS, 1.0),
                                    (FREE @ LENS, 1.7), (np.array([[0.3, 12.0], [-0.05, 1.4]]), 0.6)])
def test_ray_transfer_matches_oracle(abcd, m):
    import torch

    import chromatix_b200 as cx
    import chromatix_b200.functional as cf

    rng = np.random.default_rng(0)
    u = (rng.standard_normal((64, 48)) + 1j * rng.standard_normal((64, 48))).astype(np.complex64)
    f = cx.Field.build(torch.as_tensor(u, device="cuda"), 0.5, 0.532)
    out = cf.ray_transfer(f, abcd, 1.33, m)
    ref = O.ray_transfer(O.field_build(u.astype(np.complex128), 0.5, 0.532), abcd, 1.33, m)
    assert rel(to_np(out.u), ref.u) < 1e-5
    np.testing.assert_allclose(out.dx, np.asarray(ref.dx).reshape(np.shape(out.dx)))


def test_ray_transfer_chromatic_batched_shifted_origin():
    import torch

    import chromatix_b200 as cx
    import chromatix_b200.functional as cf

    rng = np.random.default_rng(1)
    wl = np.array([0.45, 0.55, 0.65])
    u = (rng.standard_normal((2, 40, 40, 3)) + 1j * rng.standard_normal((2, 40, 40, 3))).astype(np.complex64)
    f = cx.shift_grid(cx.ChromaticScalarField(torch.as_tensor(u, device="cuda"), 0.4, 0.0,
                                              cx.Spectrum.build((wl, np.ones(3)))), (0.8, -0.4))
    abcd = FREE @ LENS
    out = cf.ray_transfer(f, abcd, 1.0, 1.3)
    for b in range(2):
        of = O.field_build(u[b].astype(np.complex128), 0.4, (wl, np.ones(3)))
        of = of.replace(origin=np.tile([0.8, -0.4], (3, 1)))
        ref = O.ray_transfer(of, abcd, 1.0, 1.3)
        assert rel(to_np(out.u[b]), ref.u) < 1e-5


def test_ray_transfer_rejects_b_zero():
    import torch

    import chromatix_b200 as cx
    import chromatix_b200.functional as cf
    from chromatix_b200._native import CxError

    f = cx.Field.build(torch.zeros((16, 16), dtype=torch.complex64, device="cuda"), 0.5, 0.5)
    with pytest.raises(CxError, match="B != 0"):
        cf.ray_transfer(f, LENS, 1.0)
