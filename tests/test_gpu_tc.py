"""Tensor-core (tcgen05) split-FP16 DFT against an FP64 DFT.

The transform is a real GEMM on FP16 hi + lo operands with FP32 accumulation;
its relative L2 error per vector is bounded by ~2^-21 times a small factor,
so the bar is 1e-5 (the accurate mode's), checked per vector over inputs
whose magnitudes span 1e-4 .. 1e4 (each vector is scaled by a power of two
before the split)."""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _lib():
    from chromatix_b200 import _native as nat

    L = nat.lib()
    L.cx_dft_split16.restype = ctypes.c_int32
    L.cx_dft_split16.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_int32,
                                 ctypes.c_void_p, ctypes.c_void_p]
    return nat, L


@pytest.mark.parametrize("R", [16, 32, 40, 64])
@pytest.mark.parametrize("inverse", [0, 1])
def test_split16_dft_matches_fp64(R, inverse):
    import torch

    nat, L = _lib()
    rng = np.random.default_rng(R + 100 * inverse)
    B = 1000  # not a multiple of the 128-vector tile
    mag = 10.0 ** rng.uniform(-4, 4, (B, 1))
    x = ((rng.standard_normal((B, R)) + 1j * rng.standard_normal((B, R))) * mag).astype(np.complex64)
    x[7] = 0  # an all-zero vector
    xt = torch.as_tensor(x, device="cuda")
    yt = torch.full_like(xt, float("nan"))
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    nat.check(L.cx_dft_split16(xt.data_ptr(), yt.data_ptr(), R, B, inverse, status.data_ptr(),
                               torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    y = yt.cpu().numpy()
    ref = np.fft.ifft(x.astype(np.complex128), axis=1) * R if inverse else np.fft.fft(x.astype(np.complex128), axis=1)
    num = np.linalg.norm(y - ref, axis=1)
    den = np.linalg.norm(ref, axis=1)
    assert np.all(y[7] == 0)
    ok = den > 0
    err = num[ok] / den[ok]
    assert err.max() < 1e-5, err.max()


def test_split16_rejects_unsupported_length():
    import torch

    nat, L = _lib()
    xt = torch.zeros((4, 24), dtype=torch.complex64, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert L.cx_dft_split16(xt.data_ptr(), xt.data_ptr(), 24, 4, 0, status.data_ptr(), None) == nat.CX_ERR_UNSUPPORTED


@pytest.mark.parametrize("N", [1280, 1024])
def test_split16_psf_matches_fp64_oracle(N):
    """The 4f PSF with its row and column transforms on the tensor cores
    (precision "split16") against the FP64 oracle, at the headline configuration's optics
    (f_obj 8 mm, f_tube 200 mm, NA 0.6, n 1.33, 3 wavelengths, 6.5 um camera
    pitch) on 3 defocus planes: relative L2 <= 1e-5, and within 3x of the
    plain FP32 path's own error."""
    import torch

    import chromatix_b200 as cx
    import chromatix_b200.functional as cf
    from oracle import chromatix_oracle as O
    from tests.helpers import rel

    wl = np.array([0.45, 0.532, 0.63])
    dxw = 200000.0 * wl / (1.33 * N * 6.5)
    dx = np.stack([dxw, dxw], -1)
    rng = np.random.default_rng(5)
    z = np.array([-4.0, 0.3, 5.0])
    phase = rng.uniform(0, 2 * np.pi, (N, N)).astype(np.float32)

    def run(prec):
        with cx.precision(prec):
            f = cf.objective_point_source((N, N), dx, (wl, np.ones(3)), z, 8000.0, 1.33, 0.6)
            f = cf.ff_lens(cf.phase_change(f, torch.as_tensor(phase, device="cuda")), 200000.0, 1.33)
            return f.intensity.cpu().numpy()

    I16, I32 = run("split16"), run("accurate")
    assert np.isfinite(I16).all()
    O.set_fft_workers(8)
    ref = O.ff_lens(O.phase_change(O.objective_point_source((N, N), dx, (wl, np.ones(3)), z, 8000.0, 1.33, 0.6),
                                   phase), 200000.0, 1.33).intensity
    e16, e32 = rel(I16, ref), rel(I32, ref)
    assert e16 < 1e-5, (e16, e32)
    assert e16 < 3 * e32 + 1e-6, (e16, e32)


@pytest.mark.parametrize("method,mode", [("asm", "full"), ("asm", "same"), ("transfer", "full"), ("exact", "same")])
def test_split16_propagation_512_pad_256_matches_fp64(method, mode):
    """The single-field propagation configuration (512^2, pad 256 -> 1024^2,
    dx 0.3, lambda 0.532, n 1.33, z 100 um) with the column pass on the tensor
    cores, batch of 3 fields: relative L2 <= 1e-5 against the FP64 oracle."""
    import torch

    import chromatix_b200 as cx
    import chromatix_b200.functional as cf
    from oracle import chromatix_oracle as O
    from tests.helpers import oracle_field, rand_field, rel

    from chromatix_b200.core.field import ScalarField
    from chromatix_b200.core.spectrum import Spectrum

    u = np.stack([rand_field((512, 512), seed=s) for s in (1, 2, 3)])
    f = ScalarField(torch.as_tensor(u, device="cuda"), 0.3, 0.0, Spectrum.build(0.532))
    kw = dict(mode=mode)
    with cx.precision("split16"):
        if method == "transfer":
            out = cf.transfer_propagate(f, 100.0, 1.33, 256, **kw).u
        else:
            out = cf.asm_propagate(f, 100.0, 1.33, 256, remove_evanescent=(method == "exact"), **kw).u
    out = out.cpu().numpy()
    for b in range(3):
        fo = oracle_field(u[b], 0.3, 0.532)
        if method == "transfer":
            ref = O.transfer_propagate(fo, 100.0, 1.33, 256, **kw).u
        else:
            ref = O.asm_propagate(fo, 100.0, 1.33, 256, remove_evanescent=(method == "exact"), **kw).u
        e = rel(out[b], ref)
        assert e < 1e-5, (b, e)


def test_split16_propagation_1280_grid_and_adjoint():
    """A 640^2 field padded to 1280^2 (the 40 x 32 four-step) forward against
    the oracle, and the gradient (conj(H) through the same tensor-core pass)
    by the dot-product identity <A u, w> = <u, A^H w>."""
    import torch

    import chromatix_b200 as cx
    import chromatix_b200.functional as cf
    from oracle import chromatix_oracle as O
    from tests.helpers import oracle_field, rand_field, rel

    u = rand_field((640, 640), seed=9)
    ut = torch.as_tensor(u, device="cuda").requires_grad_(True)
    with cx.precision("split16"):
        y = cf.asm_propagate(cx.Field.build(ut, 0.25, 0.6), 60.0, 1.0, 320, mode="same").u
    ref = O.asm_propagate(oracle_field(u, 0.25, 0.6), 60.0, 1.0, 320, mode="same").u
    assert rel(y.detach().cpu().numpy(), ref) < 1e-5
    w = (np.random.default_rng(10).standard_normal(y.shape) + 1j).astype(np.complex64)
    torch.real(torch.sum(torch.conj(torch.as_tensor(w, device="cuda")) * y)).backward()
    lhs = np.vdot(y.detach().cpu().numpy().astype(np.complex128).ravel(), w.astype(np.complex128).ravel())
    rhs = np.vdot(u.astype(np.complex128).ravel(), ut.grad.cpu().numpy().astype(np.complex128).ravel())
    assert abs(lhs - rhs) <= 1e-5 * abs(lhs)


def test_split16_multislice_1024_forward_and_gradient():
    """Multislice at 1024^2 (the differentiable configuration's grid, 8 slices)
    with the slice loop's row and column transforms on the tensor cores,
    against the FP64 restatement.  Each slice runs four split-precision
    transforms (2-5e-7 each on the hardware) and their errors add up slice by
    slice, so the bars are depth-scaled: forward <= 5e-5 and dL/d dn <= 5e-4
    at 8 slices (the FP32 path's bars are 1e-5 / 1e-4 at any depth)."""
    import torch

    import chromatix_b200 as cx
    import chromatix_b200.functional as cf
    from oracle import chromatix_oracle as O
    from tests.helpers import cuda_field, rand_field, rel

    D, N = 8, 1024
    rng = np.random.default_rng(11)
    u = rand_field((N, N), seed=12, amp=(0.9, 1.0))
    dn = (0.02 * rng.standard_normal((D, N, N))).astype(np.float32)
    ab = rng.uniform(0, 0.05, (D, N, N)).astype(np.float32)
    target = rng.uniform(0.5, 1.5, (N, N))
    O.set_fft_workers(8)
    L64, gdn64, _, uo64 = O.multislice_loss_and_grad(u, dn.astype(np.float64), ab.astype(np.float64), target,
                                                     1.33, 0.2, 0.532, 0.1)
    dn_t = torch.as_tensor(dn, device="cuda").requires_grad_(True)
    with cx.precision("split16"):
        out = cf.multislice_thick_sample(cuda_field(u, 0.1, 0.532), torch.as_tensor(ab, device="cuda"), dn_t, 1.33,
                                         0.2, 0, checkpoint_every=4)
        loss = ((out.u.abs() ** 2 - torch.as_tensor(target, device="cuda", dtype=torch.float32)) ** 2).sum()
        loss.backward()
    e_fwd = rel(out.u.detach().cpu().numpy(), uo64)
    e_grad = rel(dn_t.grad.cpu().numpy(), gdn64)
    assert e_fwd < 5e-5, (e_fwd, e_grad)
    assert abs(float(loss) - L64) / L64 < 1e-4
    assert e_grad < 5e-4, (e_fwd, e_grad)


def test_no_tensor_core_wait_ran_out():
    """After the split-precision runs of this module (and one more PSF here),
    no CTA gave up on an MMA wait: the device counter cx_tc_timeouts reads 0,
    and a reset leaves it at 0."""
    import ctypes as C

    import torch

    import chromatix_b200 as cx
    import chromatix_b200.functional as cf
    from chromatix_b200 import _native as nat

    L = nat.lib()
    L.cx_tc_timeouts.restype = C.c_int32
    L.cx_tc_timeouts.argtypes = [C.POINTER(C.c_int32), C.c_int32]
    with cx.precision("split16"):
        f = cf.objective_point_source((1024, 1024), 0.25, 0.532, np.array([0.0, 2.0]), 8000.0, 1.33, 0.6)
        I = cf.ff_lens(f, 200000.0, 1.33).intensity
    torch.cuda.synchronize()
    assert torch.isfinite(I).all()
    n = C.c_int32(-1)
    assert L.cx_tc_timeouts(C.byref(n), 1) == 0
    assert n.value == 0
    assert L.cx_tc_timeouts(C.byref(n), 0) == 0
    assert n.value == 0
