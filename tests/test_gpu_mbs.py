"""Modified Born series on the GPU vs the FP64 oracle
(experimental/modified_born_series/solver.py:42-146): the preconditioned
source, single fixed-point updates from arbitrary iterates, and 40 iterations
of the solve, on cubic and non-cubic grids with absorbing boundaries."""

import numpy as np
import pytest

from oracle import chromatix_oracle as O
from tests.helpers import rel, to_np

pytestmark = pytest.mark.gpu

WAVELENGTH = 0.5  # um
K0 = 2 * np.pi / WAVELENGTH
SPACING = 0.1


def _problem(shape, n_sphere=1.2, seed=0, bc=4):
    """Sphere (with a weakly absorbing part) in a background of index 1, absorbing
    layers of ``bc`` voxels on every face, an x-polarised Gaussian current blob."""
    inner = tuple(s - 2 * bc for s in shape)
    g = np.stack(np.meshgrid(*[np.arange(n) - n // 2 for n in inner], indexing="ij"), -1) * SPACING
    r = np.linalg.norm(g - np.array([0.3, -0.2, 0.1])[: 3], axis=-1)
    n = np.where(r < 0.8, n_sphere + 0.01j, 1.0)
    perm, roi = O.mbs_add_absorbing_bc(n**2, SPACING, (0, 1, 2), bc * SPACING, 0.25)
    gs = np.stack(np.meshgrid(*[np.arange(s) - s // 2 for s in shape], indexing="ij"), -1) * SPACING
    rs = np.linalg.norm(gs - np.array([-0.4, 0.0, -0.5]), axis=-1)
    J = np.zeros(shape + (3,), np.complex128)
    J[..., 0] = np.exp(-(rs**2) / (2 * 0.15**2))
    rng = np.random.default_rng(seed)
    J[..., 2] = 0.3 * np.exp(-(rs**2) / (2 * 0.2**2)) * np.exp(1j * rng.uniform(0, 2 * np.pi))
    return perm, O.mbs_source_field(J, K0), roi


def _cuda_solve(perm, src_field, shift, scale, **kw):
    import torch

    from chromatix_b200.experimental import mbs

    sample = mbs.Sample(torch.as_tensor(perm.astype(np.complex64), device="cuda"), SPACING)
    source = mbs.Source(torch.zeros(perm.shape + (3,), dtype=torch.complex64, device="cuda"), K0)
    source.field = torch.as_tensor(src_field.astype(np.complex64), device="cuda")
    return mbs.solve(sample, source, shift=shift, scale=scale, return_info=True, **kw)


@pytest.mark.parametrize("shape", [(32, 32, 32), (24, 40, 32)])
def test_mbs_precondition_and_steps(shape):
    perm, src, _ = _problem(shape)
    op = O.MBSOperator(perm, SPACING, K0, src)
    # maxiter=1 from the preconditioned source: one update of prec_y
    E1, info = _cuda_solve(perm, src, op.bias, op.scale, maxiter=1, tol=0.0)
    assert abs(info["num_scale"] - op.num_scale) / op.num_scale < 1e-5
    ref1 = op.step(op.prec_y) * op.num_scale
    assert rel(to_np(E1), ref1) < 2e-5
    # an arbitrary iterate
    rng = np.random.default_rng(3)
    x0 = (rng.standard_normal(shape + (3,)) + 1j * rng.standard_normal(shape + (3,))) * op.num_scale
    import torch

    E2, _ = _cuda_solve(perm, src, op.bias, op.scale, maxiter=1, tol=0.0,
                        initial_E=torch.as_tensor(x0.astype(np.complex64), device="cuda"))
    ref2 = op.step(x0 / op.num_scale) * op.num_scale
    assert rel(to_np(E2), ref2) < 2e-5


def test_mbs_solve_iterations_track_the_oracle():
    shape = (32, 32, 32)
    perm, src, roi = _problem(shape)
    E, it, res, op = O.mbs_solve(perm, SPACING, K0, src, maxiter=40, tol=0.0)
    Eg, info = _cuda_solve(perm, src, op.bias, op.scale, maxiter=40, tol=0.0)
    assert info["iterations"] == 40
    assert rel(to_np(Eg), E) < 1e-4
    assert rel(to_np(Eg)[roi], E[roi]) < 1e-4
    assert abs(info["residual_rel"] - res) / res < 1e-2


def test_mbs_stopping_rules():
    shape = (24, 24, 24)
    perm, src, _ = _problem(shape, bc=3)
    op = O.MBSOperator(perm, SPACING, K0, src)
    _, info = _cuda_solve(perm, src, op.bias, op.scale, maxiter=500, tol=0.0, rtol=1e-3)
    assert info["residual_rel"] < 1e-3 and info["iterations"] < 500
    # the oracle reaches the same relative residual at the same iteration (+-1)
    x = op.prec_y.copy()
    for k in range(1, 501):
        xn = op.step(x)
        r = np.linalg.norm(xn - x) / np.linalg.norm(xn)
        x = xn
        if r < 1e-3:
            break
    assert abs(k - info["iterations"]) <= 1
    # absolute rule of the fixed-point iteration: ||x_{k+1} - x_k|| <= tol
    _, info = _cuda_solve(perm, src, op.bias, op.scale, maxiter=500, tol=1e-2)
    assert info["residual_abs"] <= 1e-2


def test_mbs_shift_and_scale_on_device():
    import torch

    from chromatix_b200.experimental import mbs

    perm, _, _ = _problem((32, 32, 32))
    c0, s0 = O.mbs_shift_and_scale(perm)
    c, s = mbs.get_shift_and_scale(torch.as_tensor(perm.astype(np.complex64), device="cuda"))
    R0, R = abs(1 / s0), abs(1 / s)
    assert abs(c - c0) <= 1e-4 * R0
    assert R0 * (1 - 1e-5) <= R <= R0 * (1 + 1e-3)


def test_mbs_rejects_unsupported_lengths():
    from chromatix_b200._native import CxError

    perm = np.ones((17, 32, 32), np.complex128)
    with pytest.raises(CxError):
        _cuda_solve(perm, np.zeros(perm.shape + (3,)), 1.0, 1.0, maxiter=1)


def test_mbs_bicgstab_iterates_and_converged_field():
    """use_bicgstab=True (solver.py:143-144): the first BiCGStab iterates track
    the FP64 restatement of the algorithm, and the converged field equals the
    fixed-point solution of the same preconditioned system."""
    shape = (32, 32, 32)
    perm, src, roi = _problem(shape)
    op = O.MBSOperator(perm, SPACING, K0, src)
    for k in (1, 3):
        x64, it64, _ = O.mbs_bicgstab(op, op.prec_y, maxiter=k, tol=0.0)
        Eb, info = _cuda_solve(perm, src, op.bias, op.scale, maxiter=k, tol=0.0, use_bicgstab=True)
        assert info["iterations"] == it64 == k
        assert rel(to_np(Eb), x64 * op.num_scale) < 1e-4, k
    Eb, info = _cuda_solve(perm, src, op.bias, op.scale, maxiter=400, tol=1e-6, use_bicgstab=True)
    assert info["status"] == "converged" and info["residual_rel"] <= 1e-6
    Ef, it, res, _ = O.mbs_solve(perm, SPACING, K0, src, maxiter=3000, tol=1e-9, shift=op.bias, scale=op.scale)
    assert rel(to_np(Eb), Ef) < 1e-4
    # BiCGStab needs far fewer operator applications than the fixed-point series
    assert 2 * info["iterations"] < it
