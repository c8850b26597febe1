"""Multislice forward and hand-written adjoint on the GPU vs the FP64 oracle.

Tolerances: forward relative L2 <= 1e-5 against the FP64 restatement;
gradients (dL/d dn, dL/d abs) relative L2 <= 1e-4 against the FP64 adjoint
(the loss itself is a difference of squared FP32 intensities).
"""

import numpy as np
import pytest

from oracle import chromatix_oracle as O
from tests.helpers import cuda_field, oracle_field, rand_field, rel, to_np

pytestmark = pytest.mark.gpu


def _sample(D, ny, nx, seed=0, dn_scale=0.02, ab_max=0.05):
    rng = np.random.default_rng(seed)
    dn = (dn_scale * rng.standard_normal((D, ny, nx))).astype(np.float32)
    ab = rng.uniform(0, ab_max, (D, ny, nx)).astype(np.float32)
    return dn, ab


@pytest.mark.parametrize("pad,NA,kw", [(0, None, {}), (16, 0.8, {}), (8, None, dict(remove_evanescent=True)),
                                       (0, 0.5, dict(bandlimit=True))])
def test_forward_matches_oracle(pad, NA, kw):
    import chromatix_b200.functional as cf

    ny, nx, D = 64, 96, 12
    u = rand_field((ny, nx), seed=1)
    dn, ab = _sample(D, ny, nx, seed=2)
    fc = cuda_field(u, 0.1, 0.532)
    out = cf.multislice_thick_sample(fc, ab, dn, 1.33, 0.2, pad, NA=NA, **kw)
    ref = O.multislice_thick_sample(oracle_field(u, 0.1, 0.532), ab, dn, 1.33, 0.2, pad, NA=NA, **kw)
    assert out.u.shape == ref.u.shape
    assert rel(to_np(out.u), ref.u) < 1e-5


def test_thick_sample_kats():
    """tests/test_samples.py:49-101 on the CUDA path."""
    import chromatix_b200.functional as cf

    f = cf.plane_wave((2, 2), 0.1, (0.532, 1.0), power=1.0)
    z = np.zeros((4, 2, 2))
    out = cf.multislice_thick_sample(f, z, z, 1.33, 1.0, 0)
    np.testing.assert_allclose(to_np(out.u), to_np(f.u), atol=1e-6)
    out = cf.multislice_thick_sample(f, z, np.ones_like(z) * 0.5, 1.33, 0.532, 0)
    np.testing.assert_allclose(to_np(out.power), to_np(f.power), rtol=1e-5)


@pytest.mark.parametrize("K", [0, 1, 5, 12])
def test_adjoint_matches_fp64_gradient(K):
    import torch

    import chromatix_b200.functional as cf

    ny, nx, D = 64, 64, 12
    lam, dz, n, dx = 0.532, 0.2, 1.33, 0.1
    u = rand_field((ny, nx), seed=3, amp=(0.9, 1.0))
    dn, ab = _sample(D, ny, nx, seed=4)
    target = np.random.default_rng(5).uniform(0.5, 1.5, (ny, nx))
    L64, gdn64, gab64, _ = O.multislice_loss_and_grad(u, dn.astype(np.float64), ab.astype(np.float64), target, n,
                                                      dz, lam, dx, NA=0.9)
    dn_t = torch.as_tensor(dn, device="cuda").requires_grad_(True)
    ab_t = torch.as_tensor(ab, device="cuda").requires_grad_(True)
    out = cf.multislice_thick_sample(cuda_field(u, dx, lam), ab_t, dn_t, n, dz, 0, NA=0.9, checkpoint_every=K)
    I = out.u.abs() ** 2
    loss = ((I - torch.as_tensor(target, device="cuda", dtype=torch.float32)) ** 2).sum()
    loss.backward()
    assert abs(float(loss) - L64) / L64 < 1e-4
    assert rel(to_np(dn_t.grad), gdn64) < 1e-4
    assert rel(to_np(ab_t.grad), gab64) < 1e-4


def test_adjoint_against_central_differences():
    """Central finite differences of the FP64 oracle loss vs the CUDA adjoint."""
    import torch

    import chromatix_b200.functional as cf

    ny, nx, D = 32, 32, 6
    lam, dz, n, dx = 0.532, 0.2, 1.33, 0.1
    u = rand_field((ny, nx), seed=6, amp=(0.9, 1.0))
    dn, ab = _sample(D, ny, nx, seed=7)
    target = np.random.default_rng(8).uniform(0.5, 1.5, (ny, nx))
    dn_t = torch.as_tensor(dn, device="cuda").requires_grad_(True)
    out = cf.multislice_thick_sample(cuda_field(u, dx, lam), torch.as_tensor(ab, device="cuda"), dn_t, n, dz, 0)
    loss = ((out.u.abs() ** 2 - torch.as_tensor(target, device="cuda", dtype=torch.float32)) ** 2).sum()
    loss.backward()
    g = to_np(dn_t.grad)
    rng = np.random.default_rng(9)
    h = 1e-4
    for _ in range(6):
        i, y, x = rng.integers(D), rng.integers(ny), rng.integers(nx)
        dp = dn.astype(np.float64).copy()
        dm = dp.copy()
        dp[i, y, x] += h
        dm[i, y, x] -= h
        Lp = O.multislice_loss_and_grad(u, dp, ab.astype(np.float64), target, n, dz, lam, dx)[0]
        Lm = O.multislice_loss_and_grad(u, dm, ab.astype(np.float64), target, n, dz, lam, dx)[0]
        fd = (Lp - Lm) / (2 * h)
        assert abs(g[i, y, x] - fd) <= 1e-3 * max(1.0, abs(fd)), (i, y, x, g[i, y, x], fd)


def test_field_gradient_and_batch():
    import torch

    import chromatix_b200 as cx
    import chromatix_b200.functional as cf

    ny, nx, D = 32, 64, 4
    u = rand_field((2, ny, nx), seed=10)
    dn, ab = _sample(D, ny, nx, seed=11)
    ut = torch.as_tensor(u, device="cuda").requires_grad_(True)
    f = cx.ScalarField(ut, 0.1, 0.0, cx.MonoSpectrum(0.532))
    out = cf.multislice_thick_sample(f, ab, dn, 1.33, 0.2, 0)
    assert out.u.shape == (2, ny, nx)
    for b in range(2):
        ref = O.multislice_thick_sample(oracle_field(u[b], 0.1, 0.532), ab, dn, 1.33, 0.2, 0)
        assert rel(to_np(out.u[b]), ref.u) < 1e-5
    (out.u.abs() ** 2).sum().backward()
    # the map is unitary up to absorption: d/du sum|u_out|^2 = 2 A^H A u, nonzero
    assert float(ut.grad.abs().sum()) > 0


def test_return_stack_planes_match_partial_stacks():
    """return_stack (functional/samples.py:253-260): plane k of the stack is the
    field after the first k slices (no final defocus), cropped."""
    import chromatix_b200.functional as cf

    ny, nx, D, pad = 48, 64, 5, 8
    u = rand_field((ny, nx), seed=9)
    dn, ab = _sample(D, ny, nx, seed=10)
    fc = cuda_field(u, 0.1, 0.532)
    st = cf.multislice_thick_sample(fc, ab, dn, 1.33, 0.2, pad, return_stack=True)
    assert tuple(st.u.shape) == (D, ny, nx)
    for k in (1, 3, 5):
        ref = O.multislice_thick_sample(oracle_field(u, 0.1, 0.532), ab[:k], dn[:k], 1.33, 0.2, pad,
                                        reverse_propagate_distance=0.0)
        assert rel(to_np(st.u[k - 1]), ref.u) < 1e-5


def test_gradient_independent_of_checkpoint_spacing():
    """The adjoint recomputes segment s - 1 on a second stream while it works
    through segment s (double-buffered records).  Any checkpoint spacing must
    give the gradients of a single segment (no recomputation overlap at all):
    a race between the two chains would show up as a difference here.  On a
    power-of-two grid the recomputed records are the forward's bits, so the
    gradients agree to the last bit."""
    import torch

    import chromatix_b200.functional as cf

    ny, nx, D = 128, 128, 24
    lam, dz, n, dx = 0.532, 0.2, 1.33, 0.1
    u = rand_field((ny, nx), seed=11, amp=(0.9, 1.0))
    dn, ab = _sample(D, ny, nx, seed=12)
    tgt = torch.as_tensor(np.random.default_rng(13).uniform(0.5, 1.5, (ny, nx)).astype(np.float32), device="cuda")
    grads = {}
    for K in (D, 1, 2, 5, 7):
        dn_t = torch.as_tensor(dn, device="cuda").requires_grad_(True)
        ab_t = torch.as_tensor(ab, device="cuda").requires_grad_(True)
        out = cf.multislice_thick_sample(cuda_field(u, dx, lam), ab_t, dn_t, n, dz, 0, checkpoint_every=K)
        loss = ((out.u.abs() ** 2 - tgt) ** 2).sum()
        loss.backward()
        grads[K] = (dn_t.grad.cpu().numpy(), ab_t.grad.cpu().numpy())
    for K in (1, 2, 5, 7):
        np.testing.assert_array_equal(grads[K][0], grads[D][0], err_msg=f"dL/d dn, K={K}")
        np.testing.assert_array_equal(grads[K][1], grads[D][1], err_msg=f"dL/d abs, K={K}")
