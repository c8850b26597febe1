"""Hand-written adjoints (the gradients the reference takes with jax.grad)
against the FP64 oracle.

For a map A that is linear in the field, the gradient of
L = Re(sum(conj(w) A u)) is A^H w (torch's convention for complex tensors).
Its FP64 value at pixel j is conj(<w, A e_j>), evaluated with the oracle's
forward restatement on the basis vector e_j -- the exact directional
derivative, no finite-difference step.  Nonlinear parts (intensity, phase and
refractive-index maps, the PSF's phase mask) are checked by central
differences of the FP64 oracle.

Tolerances: 2e-5 relative to the gradient's largest entry for the linear
adjoints (FP32 transforms, like the forward path's 1e-5 relative-L2 bar
measured per pixel); 1e-3 relative for central differences of losses.
"""

import numpy as np
import pytest

from oracle import chromatix_oracle as O
from tests.helpers import rand_field, rel, to_np

pytestmark = pytest.mark.gpu

TOL_LIN = 2e-5


def _rng(seed):
    return np.random.default_rng(seed)


def _randc(shape, seed):
    r = _rng(seed)
    return (r.standard_normal(shape) + 1j * r.standard_normal(shape)).astype(np.complex64)


def _fp64_adjoint_at(fwd64, w, in_shape, idxs):
    """conj(<w, A e_j>) for the flat input indices j in ``idxs``."""
    out = []
    for j in idxs:
        e = np.zeros(int(np.prod(in_shape)), dtype=np.complex128)
        e[j] = 1.0
        Ae = np.asarray(fwd64(e.reshape(in_shape)), dtype=np.complex128)
        out.append(np.sum(w.astype(np.complex128) * np.conj(Ae)))
    return np.array(out)


def _check_linear_adjoint(fwd_cuda, fwd64, u, seed, n_pix=10):
    """torch gradient of Re<w, A u> vs the FP64 adjoint at sampled pixels, plus
    the dot-product identity <A u, w> = <u, A^H w> on the whole arrays."""
    import torch

    ut = torch.as_tensor(u, device="cuda").requires_grad_(True)
    y = fwd_cuda(ut)
    w = _randc(tuple(y.shape), seed)
    wt = torch.as_tensor(w, device="cuda")
    L = torch.real(torch.sum(torch.conj(wt) * y))
    L.backward()
    g = to_np(ut.grad).reshape(-1)
    idxs = _rng(seed + 1).choice(u.size, size=n_pix, replace=False)
    ref = _fp64_adjoint_at(fwd64, w, u.shape, idxs)
    scale = np.max(np.abs(ref))
    err = np.max(np.abs(g[idxs] - ref)) / scale
    assert err < TOL_LIN, err
    # <A u, w> = <u, A^H w> on the whole arrays (float32 sums, so a loose bound)
    lhs = np.vdot(to_np(y).astype(np.complex128).reshape(-1), w.astype(np.complex128).reshape(-1))
    rhs = np.vdot(u.astype(np.complex128).reshape(-1), g.astype(np.complex128))
    assert abs(lhs - rhs) <= 1e-4 * max(abs(lhs), 1.0), (lhs, rhs)
    return g


def _field(ut, dx, spectrum):
    import chromatix_b200 as cx

    return cx.Field.build(ut, dx, spectrum)


@pytest.mark.parametrize("mode", ["full", "same"])
@pytest.mark.parametrize("method", ["asm", "transfer", "exact"])
def test_propagation_adjoint(method, mode):
    import chromatix_b200.functional as cf

    u = rand_field((40, 56), seed=1)
    z, n, pad = 30.0, 1.33, 12

    def fc(ut):
        f = _field(ut, 0.3, 0.532)
        if method == "transfer":
            return cf.transfer_propagate(f, z, n, pad, mode=mode).u
        return cf.asm_propagate(f, z, n, pad, mode=mode, remove_evanescent=(method == "exact")).u

    def f64(x):
        f = O.field_build(x, 0.3, 0.532)
        if method == "transfer":
            return O.transfer_propagate(f, z, n, pad, mode=mode).u
        return O.asm_propagate(f, z, n, pad, mode=mode, remove_evanescent=(method == "exact")).u

    _check_linear_adjoint(fc, f64, u, seed=2)


def test_asm_adjoint_with_shift_bandlimit_and_tilt():
    import chromatix_b200.functional as cf

    u = rand_field((48, 48), seed=3)
    kw = dict(shift_yx=(1.5, -2.0), bandlimit=True, kykx=(0.2, -0.1))
    fc = lambda ut: cf.asm_propagate(_field(ut, 0.25, 0.5), 200.0, 1.0, 16, **kw).u
    f64 = lambda x: O.asm_propagate(O.field_build(x, 0.25, 0.5), 200.0, 1.0, 16, **kw).u
    _check_linear_adjoint(fc, f64, u, seed=4)


def test_chromatic_and_z_broadcast_adjoint_sums_over_planes():
    """A (y x wv) field propagated to three distances at once: the gradient of
    the input sums the three planes' adjoints (the broadcast's reduction)."""
    import chromatix_b200.functional as cf

    spec = (np.array([0.45, 0.6]), np.array([1.0, 2.0]))
    u = _randc((32, 40, 2), 5)
    zs = np.array([10.0, -25.0, 60.0])
    fc = lambda ut: cf.asm_propagate(_field(ut, 0.3, spec), zs, 1.33, 8).u
    f64 = lambda x: O.asm_propagate(O.field_build(x, 0.3, spec), zs, 1.33, 8).u
    _check_linear_adjoint(fc, f64, u, seed=6)


def test_kernel_propagate_adjoint_and_propagator_gradient_refused():
    import torch

    import chromatix_b200.functional as cf

    u = rand_field((32, 48), seed=7)
    f0 = _field(torch.as_tensor(u, device="cuda"), 0.3, 0.532)
    H = cf.compute_asm_propagator(f0, 15.0, 1.33)
    H64 = O.compute_asm_propagator(O.field_build(u, 0.3, 0.532), 15.0, 1.33)
    fc = lambda ut: cf.kernel_propagate(_field(ut, 0.3, 0.532), H).u
    f64 = lambda x: O.kernel_propagate(O.field_build(x, 0.3, 0.532), H64).u
    _check_linear_adjoint(fc, f64, u, seed=8)
    Hg = H.clone().requires_grad_(True)
    with pytest.raises(NotImplementedError):
        cf.kernel_propagate(f0, Hg)


@pytest.mark.parametrize("NA,inverse", [(None, False), (0.4, False), (None, True), (0.3, True)])
def test_ff_lens_adjoint(NA, inverse):
    import chromatix_b200.functional as cf

    u = rand_field((48, 40), seed=9)
    f, n = 100.0, 1.33
    fc = lambda ut: cf.ff_lens(_field(ut, 0.5, 0.532), f, n, NA=NA, inverse=inverse).u
    f64 = lambda x: O.ff_lens(O.field_build(x, 0.5, 0.532), f, n, NA=NA, inverse=inverse).u
    _check_linear_adjoint(fc, f64, u, seed=10)


def test_df_lens_and_transform_propagate_adjoints():
    import chromatix_b200.functional as cf

    u = rand_field((32, 32), seed=11)
    fc = lambda ut: cf.df_lens(_field(ut, 0.5, 0.532), 60.0, 100.0, 1.33, NA=0.5).u
    f64 = lambda x: O.df_lens(O.field_build(x, 0.5, 0.532), 60.0, 100.0, 1.33, NA=0.5).u
    _check_linear_adjoint(fc, f64, u, seed=12)
    fc = lambda ut: cf.transform_propagate(_field(ut, 0.5, 0.532), 300.0, 1.33, 16).u
    f64 = lambda x: O.transform_propagate(O.field_build(x, 0.5, 0.532), 300.0, 1.33, 16).u
    _check_linear_adjoint(fc, f64, u, seed=13)


@pytest.mark.parametrize("axis", [-1, 0])
def test_czt_adjoint(axis):
    """y[k] = scale M_k sum_j x[j] a^-j w^jk: the adjoint is the conjugate
    transpose of that matrix, formed explicitly in FP64."""
    import torch

    from chromatix_b200.utils.czt import czt_axis

    n, m, other = 40, 56, 6
    shape = (other, n) if axis == -1 else (n, other)
    x = _randc(shape, 14)
    a = 1.01 * np.exp(0.3j)
    w = 0.999 * np.exp(-2j * np.pi / 70)
    mod_n, scale = 9, 0.7
    xt = torch.as_tensor(x, device="cuda").requires_grad_(True)
    y = czt_axis(xt, m, a, w, axis=axis, mod_n=mod_n, scale=scale)
    g_out = _randc(tuple(y.shape), 15)
    torch.real(torch.sum(torch.conj(torch.as_tensor(g_out, device="cuda")) * y)).backward()
    j = np.arange(n)[None, :]
    k = np.arange(m)[:, None]
    M = scale * (w ** (-mod_n * k) * a**mod_n) * a ** (-j.astype(float)) * w ** (j * k)  # (m, n)
    xx = np.moveaxis(x, axis, -1).astype(np.complex128)
    assert rel(np.moveaxis(to_np(y), axis, -1), xx @ M.T) < 1e-5
    gg = np.moveaxis(g_out, axis, -1).astype(np.complex128)
    ref = gg @ np.conj(M)
    assert rel(np.moveaxis(to_np(xt.grad), axis, -1), ref) < 1e-5


def test_zoomed_fft_adjoint():
    import torch

    import importlib

    C = importlib.import_module("chromatix_b200.utils.czt")

    x = _randc((24, 32), 16)
    xt = torch.as_tensor(x, device="cuda").requires_grad_(True)
    y = C.zoomed_fft(xt, -1.2, 0.9, (20, 36))
    g_out = _randc(tuple(y.shape), 17)
    torch.real(torch.sum(torch.conj(torch.as_tensor(g_out, device="cuda")) * y)).backward()
    # FP64: the zoomed FFT is separable, y = Ay x Ax^T
    def mat(nn, mm, k0, k1):
        w = np.exp(1j * (k1 - k0) / (mm - 1))
        a = np.exp(-1j * k0)
        jj = np.arange(nn)[None, :]
        kk = np.arange(mm)[:, None]
        return a ** (-jj.astype(float)) * w ** (jj * kk)
    Ay, Ax = mat(24, 20, -1.2, 0.9), mat(32, 36, -1.2, 0.9)
    assert rel(to_np(y), Ay @ x @ Ax.T) < 1e-5
    ref = np.conj(Ay).T @ g_out.astype(np.complex128) @ np.conj(Ax)
    assert rel(to_np(xt.grad), ref) < 1e-5


def test_phase_change_and_intensity_gradients_vs_central_differences():
    """L = sum((|phase_change(u, phi)|^2 ... ) through ff_lens) -- the phase
    mask and the field both get gradients; chromatic with spectral modulation."""
    import torch

    import chromatix_b200.functional as cf

    spec = (np.array([0.5, 0.62]), np.array([1.0, 1.0]))
    u = _randc((24, 24, 2), 18)
    phi = _rng(19).uniform(0, 2 * np.pi, (24, 24)).astype(np.float32)
    target = _rng(20).uniform(0, 1, (24, 24))

    def loss64(phi64, u64):
        f = O.field_build(u64, 0.4, spec)
        f = O.phase_change(f, phi64)
        f = O.ff_lens(f, 50.0, 1.0)
        I = f.intensity
        return float(np.sum((I - target) ** 2))

    phit = torch.as_tensor(phi, device="cuda").requires_grad_(True)
    ut = torch.as_tensor(u, device="cuda").requires_grad_(True)
    f = cf.phase_change(_field(ut, 0.4, spec), phit)
    f = cf.ff_lens(f, 50.0, 1.0)
    I = f.intensity
    L = torch.sum((I - torch.as_tensor(target, device="cuda", dtype=torch.float32)) ** 2)
    L.backward()
    L64 = loss64(phi.astype(np.float64), u.astype(np.complex128))
    assert abs(float(L) - L64) / L64 < 1e-4
    gphi, gu = to_np(phit.grad), to_np(ut.grad)
    h = 1e-5
    rng = _rng(21)
    for _ in range(5):
        y, x = rng.integers(24), rng.integers(24)
        pp, pm = phi.astype(np.float64).copy(), phi.astype(np.float64).copy()
        pp[y, x] += h
        pm[y, x] -= h
        fd = (loss64(pp, u.astype(np.complex128)) - loss64(pm, u.astype(np.complex128))) / (2 * h)
        assert abs(gphi[y, x] - fd) <= 1e-3 * max(abs(fd), 1e-3 * np.abs(gphi).max()), (y, x, gphi[y, x], fd)
        w = rng.integers(2)
        up, um = u.astype(np.complex128).copy(), u.astype(np.complex128).copy()
        up[y, x, w] += h
        um[y, x, w] -= h
        fdr = (loss64(phi.astype(np.float64), up) - loss64(phi.astype(np.float64), um)) / (2 * h)
        up[y, x, w] -= h - 1j * h
        um[y, x, w] += h - 1j * h
        fdi = (loss64(phi.astype(np.float64), up) - loss64(phi.astype(np.float64), um)) / (2 * h)
        ref = fdr + 1j * fdi
        assert abs(gu[y, x, w] - ref) <= 1e-3 * max(abs(ref), 1e-3 * np.abs(gu).max()), (gu[y, x, w], ref)


def test_thin_sample_gradients():
    import torch

    import chromatix_b200.functional as cf

    u = rand_field((32, 32), seed=22)
    dn = (_rng(23).standard_normal((32, 32)) * 0.05).astype(np.float32)
    ab = _rng(24).uniform(0, 0.05, (32, 32)).astype(np.float32)
    w = _randc((32, 32), 25)

    def loss64(d, a, uu):
        f = O.thin_sample(O.field_build(uu, 0.2, 0.532), a, d, 0.5)
        return float(np.real(np.sum(np.conj(w) * f.u)))

    dt = torch.as_tensor(dn, device="cuda").requires_grad_(True)
    at = torch.as_tensor(ab, device="cuda").requires_grad_(True)
    ut = torch.as_tensor(u, device="cuda").requires_grad_(True)
    out = cf.thin_sample(_field(ut, 0.2, 0.532), at, dt, 0.5).u
    ref_out = O.thin_sample(O.field_build(u, 0.2, 0.532), ab, dn, 0.5).u
    assert rel(to_np(out), ref_out) < 1e-6
    torch.real(torch.sum(torch.conj(torch.as_tensor(w, device="cuda")) * out)).backward()
    h = 1e-6
    rng = _rng(26)
    d64, a64, u64 = dn.astype(np.float64), ab.astype(np.float64), u.astype(np.complex128)
    for _ in range(5):
        y, x = rng.integers(32), rng.integers(32)
        for arr, g in ((d64, dt.grad), (a64, at.grad)):
            p, m = arr.copy(), arr.copy()
            p[y, x] += h
            m[y, x] -= h
            args_p = (p, a64, u64) if arr is d64 else (d64, p, u64)
            args_m = (m, a64, u64) if arr is d64 else (d64, m, u64)
            fd = (loss64(*args_p) - loss64(*args_m)) / (2 * h)
            assert abs(float(g[y, x]) - fd) <= 1e-3 * max(abs(fd), 1e-2), (y, x, float(g[y, x]), fd)
    # the field gradient is g conj(t)
    t = ref_out / u
    assert rel(to_np(ut.grad), w * np.conj(t)) < 1e-6


def test_psf_phase_mask_gradient_vs_central_differences():
    """The 4f PSF (objective_point_source -> phase_change -> ff_lens ->
    intensity) with a phase mask that requires a gradient: the lazy fused path
    steps aside for the differentiable chain, whose adjoints run natively."""
    import torch

    import chromatix_b200.functional as cf

    N = 48
    spec = (np.array([0.5, 0.6]), np.array([1.0, 1.0]))
    zs = np.array([-2.0, 0.0, 3.0])
    f_obj, n, NA, f_tube = 2000.0, 1.33, 0.5, 20000.0
    dxw = f_tube * spec[0] / (n * N * 6.5)
    dx = np.stack([dxw, dxw], -1)
    phi = _rng(27).uniform(0, 2 * np.pi, (N, N)).astype(np.float32)
    target = _rng(28).uniform(0, 1e-3, (3, N, N))

    def loss64(p):
        s = O.objective_point_source((N, N), dx, spec, zs, f_obj, n, NA)
        s = O.phase_change(s, p)
        s = O.ff_lens(s, f_tube, n)
        return float(np.sum((s.intensity - target) ** 2))

    pt = torch.as_tensor(phi, device="cuda").requires_grad_(True)
    src = cf.objective_point_source((N, N), dx, spec, zs, f_obj, n, NA)
    I = cf.ff_lens(cf.phase_change(src, pt), f_tube, n).intensity
    L = torch.sum((I - torch.as_tensor(target, device="cuda", dtype=torch.float32)) ** 2)
    L.backward()
    L64 = loss64(phi.astype(np.float64))
    assert abs(float(L) - L64) / L64 < 1e-4
    g = to_np(pt.grad)
    # gradient pixels inside the pupil (outside, the source is zero)
    rng = _rng(29)
    cand = np.argwhere(np.abs(g) > 1e-2 * np.abs(g).max())
    h = 1e-5
    for y, x in cand[rng.choice(len(cand), size=5, replace=False)]:
        pp, pm = phi.astype(np.float64).copy(), phi.astype(np.float64).copy()
        pp[y, x] += h
        pm[y, x] -= h
        fd = (loss64(pp) - loss64(pm)) / (2 * h)
        assert abs(g[y, x] - fd) <= 2e-3 * max(abs(fd), 1e-3 * np.abs(g).max()), (y, x, g[y, x], fd)


def test_constant_padding_cval_matches_oracle():
    """cval != 0 (core/field.py:534-549): the native pad kernel, then the fused
    propagation without loader padding; "same" crops the padding off."""
    import torch

    import chromatix_b200.functional as cf

    u = rand_field((32, 40), seed=30)
    for mode in ("full", "same"):
        out = cf.asm_propagate(_field(torch.as_tensor(u, device="cuda"), 0.3, 0.532), 20.0, 1.33, 12, cval=0.7,
                               mode=mode).u
        ref = O.asm_propagate(O.field_build(u, 0.3, 0.532), 20.0, 1.33, 12, cval=0.7, mode=mode).u
        assert rel(to_np(out), ref) < 1e-5
    out = cf.transfer_propagate(_field(torch.as_tensor(u, device="cuda"), 0.3, 0.532), 20.0, 1.33, 12,
                                cval=-0.25).u
    ref = O.transfer_propagate(O.field_build(u, 0.3, 0.532), 20.0, 1.33, 12, cval=-0.25).u
    assert rel(to_np(out), ref) < 1e-5


def test_sas_adjoint():
    import chromatix_b200.functional as cf

    u = rand_field((32, 32), seed=31)
    for z in (80.0, -80.0):
        fc = lambda ut: cf.transform_propagate_sas(_field(ut, 0.4, 0.532), z, 1.33).u
        f64 = lambda x: O.transform_propagate_sas(O.field_build(x, 0.4, 0.532), z, 1.33).u
        _check_linear_adjoint(fc, f64, u, seed=32)
