"""Lens FFTs and the fused batched 4f PSF on the GPU vs the CPU oracle."""

import numpy as np
import pytest

from oracle import chromatix_oracle as O
from tests.helpers import cuda_field, oracle_field, rand_field, rel, to_np

TOL = 1e-5
pytestmark = pytest.mark.gpu


def _psf_inputs(n=256, nz=4, seed=0):
    rng = np.random.default_rng(seed)
    wl = np.array([0.45, 0.532, 0.63])
    f_obj, f_tube, n_med, NA, cam = 8000.0, 200000.0, 1.33, 0.6, 6.5
    dx = f_tube * wl / (n_med * n * cam)  # Optical4FSystemPSF.compute_required_spacing
    z = np.sort(rng.uniform(-5, 5, nz))
    phase = rng.uniform(0, 2 * np.pi, (n, n)).astype(np.float32)
    return dict(wl=wl, f_obj=f_obj, f_tube=f_tube, n=n_med, NA=NA, dx=dx, z=z, phase=phase, shape=(n, n))


def _oracle_psf(p, prec=O.FP64, with_phase=True):
    f = O.objective_point_source(p["shape"], p["dx"], (p["wl"], np.ones(3)), p["z"], p["f_obj"], p["n"], p["NA"],
                                 prec=prec)
    if with_phase:
        f = O.phase_change(f, p["phase"])
    return O.ff_lens(f, p["f_tube"], p["n"])


def _cuda_psf(p, with_phase=True):
    import chromatix_b200.functional as cf

    f = cf.objective_point_source(p["shape"], p["dx"], (p["wl"], np.ones(3)), p["z"], p["f_obj"], p["n"], p["NA"])
    if with_phase:
        f = cf.phase_change(f, p["phase"])
    return cf.ff_lens(f, p["f_tube"], p["n"])


@pytest.mark.parametrize("with_phase", [True, False])
def test_fused_psf_intensity_matches_oracle(with_phase):
    p = _psf_inputs()
    out = _cuda_psf(p, with_phase)
    I = to_np(out.intensity)
    ref = _oracle_psf(p, with_phase=with_phase)
    Iref = ref.intensity
    assert I.shape == Iref.shape == (4, 256, 256)
    assert rel(I, Iref) < TOL
    np.testing.assert_allclose(out.dx, ref.dx, rtol=1e-12)


def test_fused_psf_1280_grid():
    """Full 1280^2 grid of the batched PSF benchmark, 2 defocus planes."""
    p = _psf_inputs(n=1280, nz=2, seed=3)
    I = to_np(_cuda_psf(p).intensity)
    O.set_fft_workers(8)
    Iref = _oracle_psf(p).intensity
    assert rel(I, Iref) < TOL


def test_materialised_psf_field_matches_oracle():
    p = _psf_inputs(n=128, nz=3, seed=1)
    out = _cuda_psf(p)
    ref = _oracle_psf(p)
    u = to_np(out.u)
    assert u.shape == ref.u.shape
    assert rel(u, ref.u) < TOL
    # eager intensity of the materialised field equals the fused intensity
    assert rel(to_np(out.intensity), ref.intensity) < TOL


def test_ref32_psf():
    """The reference-order float32 mode against the oracle's float32
    restatement (same operation order) at the 1e-5 bar, and both against FP64."""
    import chromatix_b200 as cx

    p = _psf_inputs(n=128, nz=2, seed=2)
    with cx.precision("ref32"):
        I = to_np(_cuda_psf(p).intensity)
    Iref = _oracle_psf(p, O.REF32).intensity
    I64 = _oracle_psf(p).intensity
    e, e_ref, e_ours = rel(I, Iref), rel(Iref, I64), rel(I, I64)
    assert e < 1e-5, (e, e_ref, e_ours)
    assert e_ours < 3 * e_ref + 1e-6, (e, e_ref, e_ours)


def test_point_source_power_normalisation():
    """tests/test_sources.py:70-79 on the CUDA path."""
    import chromatix_b200.functional as cf

    for power, z, shape in [(1.0, 0.5, (512, 512)), (100.0, 1.0, (256, 256))]:
        f = cf.objective_point_source(shape, 0.1, (0.532, 1.0), z, 100.0, 1.33, NA=0.8, power=power)
        assert f.shape == (*shape, 1)
        np.testing.assert_allclose(to_np(f.power), power, rtol=1e-5)


def test_ff_lens_round_trip_kat():
    """tests/test_lenses.py:6-22 on the CUDA path."""
    import chromatix_b200.functional as cf

    f1 = cf.objective_point_source((512, 512), 0.3, (0.532, 1.0), 0, f=10.0, n=1.0, NA=0.8)
    f2 = cf.ff_lens(f1, f=10.0, n=1, NA=None)
    f3 = cf.ff_lens(f2, f=10.0, n=1, NA=None)
    f2b = cf.ff_lens(f3, f=10.0, n=1, NA=None, inverse=True)
    np.testing.assert_allclose(to_np(f2.intensity), to_np(f2b.intensity), atol=1e-5)
    assert to_np(f3.u).squeeze()[256, 256] != 0.0
    o1 = O.objective_point_source((512, 512), 0.3, (0.532, 1.0), 0, f=10.0, n=1.0, NA=0.8)
    o3 = O.ff_lens(O.ff_lens(o1, 10.0, 1.0), 10.0, 1.0)
    assert rel(to_np(f3.u), o3.u) < TOL
    assert rel(to_np(f2b.u), O.ff_lens(o3, 10.0, 1.0, inverse=True).u) < TOL


def test_optical_fft_lenses_vs_oracle():
    import chromatix_b200.functional as cf

    u = rand_field((96, 160, 2), seed=4)
    spec = (np.array([0.5, 0.6]), np.array([1.0, 1.0]))
    dx = np.array([0.5, 0.6])
    fc, fo = cuda_field(u, dx, spec), oracle_field(u, dx, spec)
    for z in (250.0, -250.0):
        a = cf.optical_fft(fc, z, 1.2)
        b = O.optical_fft(fo, z, 1.2)
        assert rel(to_np(a.u), b.u) < TOL
        np.testing.assert_allclose(a.dx, b.dx, rtol=1e-12)
    a = cf.ff_lens(fc, 300.0, 1.1, NA=0.05)
    b = O.ff_lens(fo, 300.0, 1.1, NA=0.05)
    assert rel(to_np(a.u), b.u) < TOL
    a = cf.df_lens(fc, 120.0, 300.0, 1.1)
    b = O.df_lens(fo, 120.0, 300.0, 1.1)
    assert rel(to_np(a.u), b.u) < TOL


def test_transform_propagate_vs_oracle_and_kat():
    import chromatix_b200.functional as cf

    u = rand_field((128, 128), seed=5)
    fc, fo = cuda_field(u, 0.4, 0.532), oracle_field(u, 0.4, 0.532)
    for z, pw in ((80.0, 64), (-80.0, 0)):
        a = cf.transform_propagate(fc, z, 1.33, pw)
        b = O.transform_propagate(fo, z, 1.33, pw)
        assert a.u.shape == b.u.shape
        assert rel(to_np(a.u), b.u) < TOL
    # analytic square aperture (tests/test_propagate.py:36-57)
    D, z, lam, n = 40.0, 100.0, 0.532, 1.33
    for shape, pad_width in [((256, 256), (512, 512)), ((1024, 256), (256, 512))]:
        dxi = D / np.array(shape)
        field = cf.plane_wave(shape, dxi[np.newaxis], (lam, 1.0), pupil=lambda f: cf.square_pupil(f, D))
        out = cf.transform_propagate(field, z, n, pad_width=pad_width)
        I_num = to_np(out.intensity).squeeze()
        xi = to_np(out.grid).squeeze().astype(np.float64)
        I_an = np.abs(O.fresnel_square_aperture(xi, z, D, lam, n)) ** 2
        assert np.mean((I_an - I_num) ** 2) / np.mean(I_an**2) < 2e-2
        field = cf.square_pupil(cf.plane_wave(shape, dxi[np.newaxis], (lam, 1.0)), D / 10)
        back = cf.transform_propagate(cf.transform_propagate(field, z, n, 0), -z, n, 0)
        np.testing.assert_allclose(to_np(back.u), to_np(field.u), rtol=2e-5, atol=2e-6)


def test_thin_sample_kats():
    """tests/test_samples.py:9-46 on the CUDA path."""
    import chromatix_b200.functional as cf

    f = cf.plane_wave((2, 2), 0.1, (0.532, 1.0), power=1.0)
    z0 = np.zeros((2, 2))
    np.testing.assert_allclose(to_np(cf.thin_sample(f, z0, z0, 1.0).u), to_np(f.u), atol=1e-7)
    out = cf.thin_sample(f, z0, np.ones((2, 2)) * 0.5, 0.532)
    np.testing.assert_allclose(to_np(out.u), -to_np(f.u), atol=1e-6)
    out = cf.thin_sample(f, np.ones((2, 2)) / (2 * np.pi), z0, 0.532)
    np.testing.assert_allclose(to_np(out.u) * np.e, to_np(f.u), rtol=1e-5)


@pytest.mark.parametrize("nz,pinned", [(64, True), (7, False), (1, True)])
def test_psf_streamed_to_host_equals_device_result(nz, pinned):
    """intensity_to(host buffer): grouped device->host copies on a side stream
    give exactly the device result (same kernels, same chunks per plane)."""
    import torch

    p = _psf_inputs(n=256, nz=nz, seed=5)
    f = _cuda_psf(p)
    dev = f.intensity.cpu()
    shape = (nz, 256, 256) if nz > 1 else (256, 256)
    host = torch.full(shape, float("nan"), dtype=torch.float32)
    if pinned:
        host = host.pin_memory()
    out = f.intensity_to(host)
    torch.cuda.current_stream().synchronize()
    assert out is host
    assert torch.equal(host, dev)
    with pytest.raises(ValueError):
        f.intensity_to(torch.empty((3, 3), dtype=torch.float32))


def test_transform_propagate_sas_vs_oracle_and_kat():
    """transform_propagate_sas (functional/propagation.py:85-165), both signs of
    z, against the FP64 oracle; the analytic square aperture
    (tests/test_propagate.py:60-76)."""
    import chromatix_b200.functional as cf

    u = rand_field((128, 96), seed=7)
    fc, fo = cuda_field(u, 0.4, 0.532), oracle_field(u, 0.4, 0.532)
    for z in (150.0, -150.0):
        a = cf.transform_propagate_sas(fc, z, 1.33)
        b = O.transform_propagate_sas(fo, z, 1.33)
        assert a.u.shape == b.u.shape
        assert rel(to_np(a.u), b.u) < TOL, z
        np.testing.assert_allclose(a.dx, b.dx, rtol=1e-12)
    H = cf.compute_sas_precompensation(fc, 150.0, 1.33)
    Ho = O.compute_sas_precompensation(fo, 150.0, 1.33)
    assert rel(to_np(H), Ho) < TOL
    D, z, lam, n = 40.0, 100.0, 0.532, 1.33
    for shape in ((256, 256), (1024, 256)):
        dxi = D / np.array(shape)
        field = cf.plane_wave(shape, dxi[np.newaxis], (lam, 1.0), pupil=lambda f: cf.square_pupil(f, D))
        out = cf.transform_propagate_sas(field, z, n)
        I_num = to_np(out.intensity).squeeze()
        xi = to_np(out.grid).squeeze().astype(np.float64)
        I_an = np.abs(O.fresnel_square_aperture(xi, z, D, lam, n)) ** 2
        assert np.mean((I_an - I_num) ** 2) / np.mean(I_an**2) < 2e-2
