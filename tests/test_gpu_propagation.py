"""CUDA propagation path vs the CPU oracle (same seeded inputs).

Tolerances (relative L2):
* accurate mode vs the FP64 oracle: 1e-5 (the stated target);
* ref32 mode vs the oracle's float32 reference-order restatement: 1e-5.
"""

import numpy as np
import pytest

from oracle import chromatix_oracle as O
from tests.helpers import cuda_field, oracle_field, rand_field, rel, to_np

TOL = 1e-5

pytestmark = pytest.mark.gpu


def _both(u, dx, spec, fn_cuda, fn_oracle, prec="accurate"):
    import chromatix_b200 as cx

    with cx.precision(prec):
        out = fn_cuda(cuda_field(u, dx, spec))
    ref = fn_oracle(oracle_field(u, dx, spec, O.FP64 if prec == "accurate" else O.REF32))
    return out, ref


@pytest.mark.parametrize("prec", ["accurate", "ref32"])
@pytest.mark.parametrize("method", ["asm", "transfer", "exact"])
@pytest.mark.parametrize("mode", ["full", "same"])
def test_single_field_512_pad_256(method, mode, prec):
    """Single 512^2 field, 0.3 um spacing, 0.532 um, n=1.33, z=100 um, padded to 1024^2."""
    import chromatix_b200.functional as cf

    u = rand_field((512, 512), seed=1)
    kw = dict(mode=mode)
    if method == "asm":
        fc = lambda f: cf.asm_propagate(f, 100.0, 1.33, 256, **kw)
        fo = lambda f: O.asm_propagate(f, 100.0, 1.33, 256, **kw)
    elif method == "exact":
        fc = lambda f: cf.asm_propagate(f, 100.0, 1.33, 256, remove_evanescent=True, **kw)
        fo = lambda f: O.asm_propagate(f, 100.0, 1.33, 256, remove_evanescent=True, **kw)
    else:
        fc = lambda f: cf.transfer_propagate(f, 100.0, 1.33, 256, **kw)
        fo = lambda f: O.transfer_propagate(f, 100.0, 1.33, 256, **kw)
    out, ref = _both(u, 0.3, 0.532, fc, fo, prec)
    assert out.u.shape == ref.u.shape
    err = rel(to_np(out.u), ref.u)
    assert err < TOL, err


def test_accurate_mode_beats_float32_reference_error():
    """The accurate path sits far closer to FP64 than the reference's float32 path."""
    import chromatix_b200.functional as cf

    u = rand_field((512, 512), seed=2)
    out = cf.asm_propagate(cuda_field(u, 0.3, 0.532), 100.0, 1.33, 256)
    f64 = O.asm_propagate(oracle_field(u, 0.3, 0.532), 100.0, 1.33, 256).u
    r32 = O.asm_propagate(oracle_field(u, 0.3, 0.532, O.REF32), 100.0, 1.33, 256).u
    e_ours = rel(to_np(out.u), f64)
    e_ref = rel(r32, f64)
    assert e_ours < TOL and e_ours < e_ref / 10, (e_ours, e_ref)


@pytest.mark.parametrize("prec", ["accurate", "ref32"])
def test_z_batch_and_large_z(prec):
    import chromatix_b200.functional as cf

    u = rand_field((256, 256), seed=3)
    z = np.array([1.0, 37.5, 500.0])
    out, ref = _both(u, 0.3, 0.45, lambda f: cf.asm_propagate(f, z, 1.33, 128, mode="same"),
                     lambda f: O.asm_propagate(f, z, 1.33, 128, mode="same"), prec)
    assert out.u.shape == (3, 256, 256)
    assert rel(to_np(out.u), ref.u) < TOL


def test_negative_z_and_evanescent_decay():
    import chromatix_b200.functional as cf

    u = rand_field((128, 256), seed=4)
    for z in (-20.0, 3.0):
        out, ref = _both(u, 0.1, 0.532, lambda f: cf.asm_propagate(f, z, 1.0, (64, 32)),
                         lambda f: O.asm_propagate(f, z, 1.0, (64, 32)))
        assert rel(to_np(out.u), ref.u) < TOL


def test_chromatic_field_per_wavelength_spacing():
    import chromatix_b200.functional as cf

    u = rand_field((96, 160, 3), seed=5)
    spec = (np.array([0.45, 0.532, 0.63]), np.array([1.0, 2.0, 1.0]))
    dx = np.array([0.2, 0.25, 0.3])
    for fn in ("asm_propagate", "transfer_propagate"):
        out, ref = _both(u, dx, spec, lambda f: getattr(cf, fn)(f, 40.0, 1.33, 80),
                         lambda f: getattr(O, fn)(f, 40.0, 1.33, 80))
        assert out.u.shape == ref.u.shape == (256, 320, 3)
        assert rel(to_np(out.u), ref.u) < TOL


def test_shift_kykx_bandlimit():
    import chromatix_b200.functional as cf

    u = rand_field((256, 256), seed=6)
    for kw in (dict(shift_yx=(3.0, -5.0)), dict(kykx=(0.2, -0.1)), dict(bandlimit=True),
               dict(bandlimit=True, shift_yx=(4.0, 2.0))):
        out, ref = _both(u, 0.3, 0.532, lambda f: cf.asm_propagate(f, 150.0, 1.33, 128, **kw),
                         lambda f: O.asm_propagate(f, 150.0, 1.33, 128, **kw))
        assert rel(to_np(out.u), ref.u) < TOL, kw
        np.testing.assert_allclose(out.origin, ref.origin)


def test_ragged_shape_and_tuple_pad():
    """(1024, 256) with pad (256, 512): a 1536 x 1280 transform."""
    import chromatix_b200.functional as cf

    u = rand_field((1024, 256, 1), seed=7)
    dx = np.array([[40.0 / 1024, 40.0 / 256]])
    out, ref = _both(u, dx, (0.532, 1.0), lambda f: cf.transfer_propagate(f, 100.0, 1.33, (256, 512), mode="same"),
                     lambda f: O.transfer_propagate(f, 100.0, 1.33, (256, 512), mode="same"))
    assert rel(to_np(out.u), ref.u) < TOL


def test_tiny_fields():
    import chromatix_b200.functional as cf

    for shape in [(2, 2), (4, 6), (5, 10), (3, 12)]:
        u = rand_field(shape, seed=8)
        out, ref = _both(u, 0.1, 0.532, lambda f: cf.asm_propagate(f, 1.0, 1.33, 0),
                         lambda f: O.asm_propagate(f, 1.0, 1.33, 0))
        assert rel(to_np(out.u), ref.u) < TOL, shape


def test_propagators_and_kernel_propagate():
    import torch

    import chromatix_b200.functional as cf

    u = rand_field((128, 128), seed=9)
    fo = oracle_field(u, 0.3, 0.532)
    fc = cuda_field(u, 0.3, 0.532)
    H = cf.compute_asm_propagator(fc, 50.0, 1.33)
    Ho = O.compute_asm_propagator(fo, 50.0, 1.33)
    assert rel(to_np(H), Ho) < TOL
    Ht = cf.compute_transfer_propagator(fc, np.array([10.0, 20.0]), 1.33)
    Hto = O.compute_transfer_propagator(fo, np.array([10.0, 20.0]), 1.33)
    assert Ht.shape == Hto.shape
    assert rel(to_np(Ht), Hto) < TOL
    out = cf.kernel_propagate(fc, Ht)
    ref = O.kernel_propagate(fo, Hto)
    assert out.u.shape == ref.u.shape
    assert rel(to_np(out.u), ref.u) < TOL
    # explicit propagator given as a numpy array
    out2 = cf.kernel_propagate(fc, Ho)
    assert rel(to_np(out2.u), O.kernel_propagate(fo, Ho).u) < TOL
    assert isinstance(out2.u, torch.Tensor)


def test_analytic_square_aperture_through_cuda():
    """tests/test_propagate.py:79-193 (analytic Fresnel KAT) on the CUDA path."""
    import chromatix_b200 as cx
    import chromatix_b200.functional as cf

    D, z, lam, n = 40.0, 100.0, 0.532, 1.33
    for shape, pad_width in [((256, 256), (512, 512)), ((1024, 256), (256, 512))]:
        dxi = D / np.array(shape)
        field = cf.plane_wave(shape, dxi[np.newaxis], (lam, 1.0), pupil=lambda f: cf.square_pupil(f, D))
        for fn, kw in [(cf.transfer_propagate, {}), (cf.asm_propagate, {}),
                       (cf.asm_propagate, dict(remove_evanescent=True)), (cf.asm_propagate, dict(bandlimit=True))]:
            out = fn(field, z, n, pad_width=pad_width, mode="same", **kw)
            I_num = to_np(out.intensity).squeeze()
            xi = to_np(out.grid).squeeze().astype(np.float64)
            I_an = np.abs(O.fresnel_square_aperture(xi, z, D, lam, n)) ** 2
            assert np.mean((I_an - I_num) ** 2) / np.mean(I_an**2) < 2e-2
    # round trip (tests/test_propagate.py:127-149)
    shape = (256, 256)
    dxi = D / np.array(shape)
    field = cf.square_pupil(cf.plane_wave(shape, dxi[np.newaxis], (lam, 1.0)), D / 10)
    fwd = cf.asm_propagate(field, z, n, 0, remove_evanescent=True)
    back = cf.asm_propagate(fwd, -z, n, 0, remove_evanescent=True)
    np.testing.assert_allclose(to_np(back.u), to_np(field.u), rtol=2e-5, atol=2e-6)
    del cx


@pytest.mark.parametrize("shape,pad,mode", [((11, 13), 0, "full"), ((11, 13), 3, "same"), ((37, 50), 5, "full")])
def test_general_lengths_through_chirp_z_transforms(shape, pad, mode):
    """Padded grids outside the fused passes' lengths (here 11 x 13, 17 x 19,
    47 x 60) propagate through chirp-Z DFTs (the reference's jnp.fft takes any
    length): FP64 oracle parity, chromatic and z-batched, and the gradient
    identity <A u, w> = <u, A^H w>."""
    import torch

    import chromatix_b200.functional as cf

    u = rand_field(shape, seed=10)
    out = cf.asm_propagate(cuda_field(u, 0.1, 0.5), 1.0, 1.0, pad, mode=mode)
    ref = O.asm_propagate(oracle_field(u, 0.1, 0.5), 1.0, 1.0, pad, mode=mode)
    assert out.u.shape == ref.u.shape
    assert rel(to_np(out.u), ref.u) < 1e-5
    out = cf.transfer_propagate(cuda_field(u, 0.1, 0.5), 2.0, 1.0, pad, mode=mode)
    ref = O.transfer_propagate(oracle_field(u, 0.1, 0.5), 2.0, 1.0, pad, mode=mode)
    assert rel(to_np(out.u), ref.u) < 1e-5
    spec = (np.array([0.5, 0.6]), np.array([1.0, 1.0]))
    uc = np.stack([u, np.conj(u)], -1).astype(np.complex64)
    zs = np.array([0.5, 1.5, 3.0])
    out = cf.asm_propagate(cuda_field(uc, 0.1, spec), zs, 1.0, pad, mode=mode)
    ref = O.asm_propagate(oracle_field(uc, 0.1, spec), zs, 1.0, pad, mode=mode)
    assert out.u.shape == ref.u.shape
    assert rel(to_np(out.u), ref.u) < 1e-5
    ut = torch.as_tensor(u, device="cuda").requires_grad_(True)
    import chromatix_b200 as cx

    y = cf.asm_propagate(cx.Field.build(ut, 0.1, 0.5), 1.0, 1.0, pad, mode=mode).u
    w = (np.random.default_rng(3).standard_normal(tuple(y.shape)) + 1j).astype(np.complex64)
    torch.real(torch.sum(torch.conj(torch.as_tensor(w, device="cuda")) * y)).backward()
    lhs = np.vdot(to_np(y).astype(np.complex128).ravel(), w.astype(np.complex128).ravel())
    rhs = np.vdot(u.astype(np.complex128).ravel(), to_np(ut.grad).astype(np.complex128).ravel())
    assert abs(lhs - rhs) <= 1e-5 * abs(lhs)


def test_published_hires_band_limited_asm_8192():
    """The reference's high-resolution example (docs/examples/
    rescaled_propagation.ipynb): a 4096^2 field padded by 2048 to an 8192^2
    transform, band-limited ASM, mode "same", against the FP64 oracle (64M
    points, computed on all host cores)."""
    import chromatix_b200.functional as cf

    u = rand_field((4096, 4096), seed=31)
    out = cf.asm_propagate(cuda_field(u, 0.3, 0.532), 400.0, 1.33, 2048, bandlimit=True, mode="same")
    assert out.u.shape == (4096, 4096)
    import os

    O.set_fft_workers(os.cpu_count())
    ref = O.asm_propagate(oracle_field(u, 0.3, 0.532), 400.0, 1.33, 2048, bandlimit=True, mode="same").u
    O.set_fft_workers(None)
    got = to_np(out.u)
    assert rel(got, ref) < 1e-5


def test_largest_grid_4096():
    """The largest compiled 2D length: a 2048^2 field padded to 4096^2 (ASM, full)."""
    import chromatix_b200.functional as cf

    u = rand_field((2048, 2048), seed=21)
    out = cf.asm_propagate(cuda_field(u, 0.3, 0.532), 200.0, 1.33, 1024)
    O.set_fft_workers(8)
    ref = O.asm_propagate(oracle_field(u, 0.3, 0.532), 200.0, 1.33, 1024)
    assert out.u.shape == ref.u.shape == (4096, 4096)
    assert rel(to_np(out.u), ref.u) < 1e-5


@pytest.mark.parametrize("boundary", ["tukey", "super_gaussian"])
def test_absorbing_boundary_is_a_no_op_like_the_reference(boundary):
    """kernel_propagate builds the tapered pupil on the pre-propagation field and
    then returns field.replace(u=u) with the unmasked propagated u
    (functional/propagation.py:460-463): the output does not change."""
    import torch

    import chromatix_b200.functional as cf

    u = rand_field((128, 128), seed=11)
    f = cuda_field(u, 0.3, 0.532)
    for fn in (cf.asm_propagate, cf.transfer_propagate):
        a = fn(f, 40.0, 1.33, 64).u
        b = fn(f, 40.0, 1.33, 64, absorbing_boundary=boundary, absorbing_boundary_width=0.5).u
        torch.cuda.synchronize()
        assert torch.equal(a, b)
    H = cf.compute_asm_propagator(f, 40.0, 1.33)
    a = cf.kernel_propagate(f, H).u
    b = cf.kernel_propagate(f, H, absorbing_boundary=boundary).u
    torch.cuda.synchronize()
    assert torch.equal(a, b)


@pytest.mark.parametrize("mode", ["full", "same"])
def test_batch_matches_lone_fields_and_adjoint(mode):
    """A batch of 12 fields (512^2, pad 256) in one call: every field equals
    its lone propagation bit for bit (planes are independent work units), and
    the batch's gradient equals the lone fields' gradients."""
    import torch

    from chromatix_b200.core.field import ScalarField
    from chromatix_b200.core.spectrum import Spectrum
    import chromatix_b200.functional as cf

    B = 12
    u = np.stack([rand_field((512, 512), seed=40 + b) for b in range(B)])
    ut = torch.as_tensor(u, device="cuda")
    spec = Spectrum.build(0.532)
    batch = cf.asm_propagate(ScalarField(ut, 0.3, 0.0, spec), 50.0, 1.33, 256, mode=mode).u
    for b in (0, 4, 5, 11):
        lone = cf.asm_propagate(ScalarField(ut[b], 0.3, 0.0, spec), 50.0, 1.33, 256, mode=mode).u
        assert torch.equal(batch[b], lone), b
    ref = O.asm_propagate(oracle_field(u[7], 0.3, 0.532), 50.0, 1.33, 256, mode=mode).u
    assert rel(to_np(batch[7]), ref) < 1e-5
    ug = ut.clone().requires_grad_(True)
    y = cf.asm_propagate(ScalarField(ug, 0.3, 0.0, spec), 50.0, 1.33, 256, mode=mode).u
    w = torch.as_tensor((np.random.default_rng(2).standard_normal(tuple(y.shape)) + 0.5j).astype(np.complex64),
                        device="cuda")
    torch.real(torch.sum(torch.conj(w) * y)).backward()
    for b in (3, 10):
        u1 = ut[b].clone().requires_grad_(True)
        y1 = cf.asm_propagate(ScalarField(u1, 0.3, 0.0, spec), 50.0, 1.33, 256, mode=mode).u
        torch.real(torch.sum(torch.conj(w[b]) * y1)).backward()
        assert torch.equal(ug.grad[b], u1.grad), b


@pytest.mark.parametrize("n,pad", [(400, 312), (514, 255), (384, 320)])
def test_first_stage_band_pruning_edges(n, pad):
    """1024-point padded grids: data inside the central half [256, 768)
    (400 + 2*312, 384 + 2*320) take the pruned first stage; 514 + 2*255 puts
    the data on [255, 769), one row and column past the band, and takes the
    unpruned transforms.  All match the FP64 oracle at 1e-5, full and same."""
    import chromatix_b200.functional as cf

    u = rand_field((n, n), seed=n + pad)
    for mode in ("full", "same"):
        out = cf.asm_propagate(cuda_field(u, 0.3, 0.532), 80.0, 1.33, pad, mode=mode)
        ref = O.asm_propagate(oracle_field(u, 0.3, 0.532), 80.0, 1.33, pad, mode=mode)
        assert out.u.shape == ref.u.shape
        assert rel(to_np(out.u), ref.u) < 1e-5, (n, pad, mode)


def test_propagation_replays_from_a_cuda_graph():
    """asm_propagate captured in a torch CUDA graph (after one warm call, so
    its plan and device plane table are cached) and replayed on new input
    data gives the eager result bit for bit."""
    import torch

    import chromatix_b200.functional as cf
    from chromatix_b200.core.field import ScalarField
    from chromatix_b200.core.spectrum import Spectrum

    spec = Spectrum.build(0.532)
    u_static = torch.as_tensor(rand_field((256, 256), seed=71), device="cuda")
    f = ScalarField(u_static, 0.3, 0.0, spec)
    cf.asm_propagate(f, 40.0, 1.33, 128)  # warm: plan, table, workspace size
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            out = cf.asm_propagate(f, 40.0, 1.33, 128).u
    torch.cuda.current_stream().wait_stream(s)
    for seed in (72, 73):
        new = torch.as_tensor(rand_field((256, 256), seed=seed), device="cuda")
        u_static.copy_(new)
        g.replay()
        torch.cuda.synchronize()
        eager = cf.asm_propagate(ScalarField(new, 0.3, 0.0, spec), 40.0, 1.33, 128).u
        assert torch.equal(out, eager), seed
