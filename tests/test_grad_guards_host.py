"""Operations without an adjoint refuse inputs that require a gradient instead
of silently cutting them from the autograd graph (no GPU: the check runs
before any device work)."""

import numpy as np
import pytest
import torch

from chromatix_b200 import _native as nat


def test_wants_grad_follows_autograd_state():
    t = torch.zeros(3, requires_grad=True)
    assert nat.wants_grad(t)
    assert not nat.wants_grad(t.detach())
    assert not nat.wants_grad(None, 1.0, np.zeros(2))
    with torch.no_grad():
        assert not nat.wants_grad(t)
        nat.refuse_grad("op", t)  # allowed: nothing is recorded
    with pytest.raises(NotImplementedError, match="no gradient"):
        nat.refuse_grad("op", t)


def test_fourier_convolution_refuses_gradients():
    from chromatix_b200.ops.convolution import fourier_convolution

    img = torch.zeros((8, 8), requires_grad=True)
    with pytest.raises(NotImplementedError):
        fourier_convolution(img, torch.zeros((3, 3)))


def test_mbs_solve_refuses_gradients():
    from chromatix_b200.experimental import mbs

    class S:
        permittivity = torch.ones((4, 4, 4), dtype=torch.complex64, requires_grad=True)

    class J:
        field = torch.zeros((4, 4, 4, 3), dtype=torch.complex64)

    with pytest.raises(NotImplementedError):
        mbs.solve(S(), J())
