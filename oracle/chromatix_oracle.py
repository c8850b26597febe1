"""CPU oracle: a numpy restatement of Chromatix's FFT-propagation hot path.

TEST INFRASTRUCTURE ONLY.  This module is the checker for the CUDA product
path: only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` may import it.  The product package
``chromatix_b200`` never imports, calls or falls back to it.

Two precision flavours of every function:

* ``"fp64"``  -- float64/complex128 throughout: the accuracy truth.
* ``"ref32"`` -- float32/complex64 evaluated in the reference's operation order
  (Python scalars are weak-typed, as in JAX), standing in for Chromatix's own
  JAX float32 path, which cannot run here (``jax`` is not installed).

Parity status: the reference's JAX path is not runnable in this environment,
so the restatement is pinned by the reference's own known-answer tests
(analytic square-aperture Fresnel field ``tests/test_propagate.py:17-33``,
propagation round trips ``tests/test_propagate.py:53-57,127-149``, thin/thick
sample identity / pi flip / 1/e ``tests/test_samples.py:9-101``, ``ff_lens``
inverse ``tests/test_lenses.py:6-22``, CZT = DFT / IDFT / ``scipy.signal.czt``
``tests/test_czt.py:15-55``, source power normalisation
``tests/test_sources.py:10-79``) -- see ``tests/test_oracle_kat.py`` and the
fixtures under ``tests/golden/``.  Bit-level parity with XLA's float32 FFT and
``jnp.fft.fftfreq`` is unpinned (third-party code, not vendored).

Every function cites the reference file:line it restates (paths relative to
the chromatix repository root, ``src/chromatix/...``).
"""

from __future__ import annotations

import dataclasses
from typing import Optional, Sequence

import numpy as np
import scipy.fft as sfft

# ---------------------------------------------------------------------------
# precision flavours
# ---------------------------------------------------------------------------


class Prec:
    """Precision flavour: ``Prec("fp64")`` or ``Prec("ref32")``."""

    def __init__(self, name: str = "fp64"):
        if name not in ("fp64", "ref32"):
            raise ValueError(f"unknown precision {name!r}")
        self.name = name
        self.real = np.float64 if name == "fp64" else np.float32
        self.cplx = np.complex128 if name == "fp64" else np.complex64

    def r(self, x):
        return np.asarray(x, dtype=self.real)

    def c(self, x):
        return np.asarray(x, dtype=self.cplx)


FP64 = Prec("fp64")
REF32 = Prec("ref32")

_WORKERS = None  # scipy.fft worker count (None = 1 thread; set by callers)


def set_fft_workers(n: Optional[int]) -> None:
    """Thread count used by the oracle's FFTs (scipy.fft ``workers``)."""
    global _WORKERS
    _WORKERS = n


def _fft2(x, axes):
    return sfft.fft2(x, axes=axes, workers=_WORKERS)


def _ifft2(x, axes):
    return sfft.ifft2(x, axes=axes, workers=_WORKERS)


def _fftn(x, axes):
    return sfft.fftn(x, axes=axes, workers=_WORKERS)


def _ifftn(x, axes):
    return sfft.ifftn(x, axes=axes, workers=_WORKERS)


# ---------------------------------------------------------------------------
# Spectrum  (core/spectrum.py:10-107)
# ---------------------------------------------------------------------------


@dataclasses.dataclass
class Spectrum:
    """Wavelengths and normalised spectral density (core/spectrum.py:10-35)."""

    wavelength: np.ndarray
    density: np.ndarray
    mono: bool = False

    @property
    def size(self) -> int:
        return int(self.wavelength.size)

    @property
    def central_wavelength(self):
        # core/spectrum.py:75-83
        return self.wavelength[0]

    @property
    def spectral_modulation(self):
        # core/spectrum.py:88-90
        return self.central_wavelength / self.wavelength


def build_spectrum(spectrum, prec: Prec = FP64) -> Spectrum:
    """``Spectrum.build`` (core/spectrum.py:37-73)."""
    if isinstance(spectrum, Spectrum):
        return spectrum
    if isinstance(spectrum, (float, int)):
        return Spectrum(prec.r([spectrum]), prec.r([1.0]), mono=True)
    if isinstance(spectrum, (tuple, list)):
        wl = np.atleast_1d(prec.r(spectrum[0]))
        dens = np.atleast_1d(prec.r(spectrum[1]))
        dens = dens / dens.sum()
        return Spectrum(wl, dens.astype(prec.real), mono=False)
    arr = np.asarray(spectrum)
    if arr.size == 1:
        return Spectrum(prec.r(arr.reshape(1)), prec.r([1.0]), mono=True)
    wl = prec.r(arr)
    return Spectrum(wl, np.full_like(wl, 1.0 / wl.size), mono=False)


# ---------------------------------------------------------------------------
# Field  (core/field.py:49-740; scalar fields only)
# ---------------------------------------------------------------------------


@dataclasses.dataclass
class OField:
    """Scalar field container mirroring ``ScalarField`` / ``ChromaticScalarField``.

    ``u`` is ``(... y x)`` for a monochromatic field (``spectrum.mono``) and
    ``(... y x wv)`` for a chromatic one (core/field.py:616-740).  ``dx`` is
    ``(2,)`` (mono) or ``(wv, 2)`` (chromatic).
    """

    u: np.ndarray
    dx: np.ndarray
    spectrum: Spectrum
    origin: np.ndarray
    prec: Prec = FP64

    # -- layout -----------------------------------------------------------
    @property
    def chromatic(self) -> bool:
        return not self.spectrum.mono

    @property
    def spatial_dims(self):
        return (-3, -2) if self.chromatic else (-2, -1)

    @property
    def spatial_shape(self):
        d = self.spatial_dims
        return (self.u.shape[d[0]], self.u.shape[d[1]])

    def replace(self, **kw) -> "OField":
        return dataclasses.replace(self, **kw)

    # -- grids (core/field.py:23-46, 640-646, 693-718) ---------------------
    @property
    def broadcasted_wavelength(self):
        # utils/shapes.py:26-43
        wl = self.spectrum.wavelength
        if wl.size > 1:
            return wl.reshape((1, 1, wl.size))
        return wl.reshape(())

    def _dx_wv(self):
        """dx as (wv, 2) (or (1, 2) for mono)."""
        return self.dx.reshape(-1, 2)

    @property
    def grid(self):
        ny, nx = self.spatial_shape
        p = self.prec
        gy = p.r(np.linspace(0, ny - 1, ny)) - p.r(ny / 2)
        gx = p.r(np.linspace(0, nx - 1, nx)) - p.r(nx / 2)
        gy = gy.astype(p.real)
        gx = gx.astype(p.real)
        GY, GX = np.meshgrid(gy, gx, indexing="ij")
        g = np.stack([GY, GX], axis=-1)  # (y x 2)
        dxw = self._dx_wv()  # (wv 2)
        grid = dxw[:, None, None, :] * g[None]  # (wv y x 2)
        org = self.origin.reshape(-1, 2)
        if self.chromatic:
            return np.moveaxis(grid, 0, 2) + org  # (y x wv 2)
        return grid[0] + org[0]

    @property
    def f_grid(self):
        return freq_grid(self.spatial_shape, self._dx_wv(), self.prec, self.chromatic)

    @property
    def k_grid(self):
        return self.prec.r(2 * np.pi) * self.f_grid

    @property
    def extent(self):
        # core/field.py:212-219
        return self.dx * self.prec.r(np.asarray(self.spatial_shape))

    @property
    def df(self):
        # core/field.py:231-239
        return self.prec.r(1.0) / self.extent

    # -- readouts (core/field.py:656-665, 728-740) -------------------------
    @property
    def intensity(self):
        if self.chromatic:
            dens = self.spectrum.density
            dens = dens.reshape((1, 1, dens.size)) if dens.size > 1 else dens.reshape(())
            return np.sum(dens * np.abs(self.u) ** 2, axis=-1)
        return np.abs(self.u) ** 2

    @property
    def power(self):
        area = np.prod(self.dx, axis=-1)
        pd = np.sum(self.intensity, axis=(-2, -1))
        if self.chromatic:
            pd = pd[..., None, None, None]
        else:
            pd = pd[..., None, None]
        return area * pd


def freq_grid(shape, dxw, prec: Prec, chromatic: bool):
    """``freq_grid`` (core/field.py:36-46): ``fftshift(fftfreq(N)) / dx``.

    ``fftfreq`` follows jax's evaluation ``k / (d * n)`` in the working dtype.
    """
    ny, nx = shape
    fy = np.fft.fftshift(_fftfreq(ny, prec))
    fx = np.fft.fftshift(_fftfreq(nx, prec))
    FY, FX = np.meshgrid(fy, fx, indexing="ij")
    g = np.stack([FY, FX], axis=-1)  # (y x 2)
    dk = prec.r(1.0) / dxw  # (wv 2)
    out = dk[:, None, None, :] * g[None]
    if chromatic:
        return np.moveaxis(out, 0, 2)  # (y x wv 2)
    return out[0]


def _fftfreq(n: int, prec: Prec):
    k = np.empty(n, dtype=prec.real)
    if n % 2 == 0:
        k[: n // 2] = np.arange(0, n // 2)
        k[n // 2 :] = np.arange(-(n // 2), 0)
    else:
        k[: (n - 1) // 2 + 1] = np.arange(0, (n - 1) // 2 + 1)
        k[(n - 1) // 2 + 1 :] = np.arange(-((n - 1) // 2), 0)
    return (k / prec.real(n)).astype(prec.real)


def field_build(u, dx, spectrum, prec: Prec = FP64) -> OField:
    """``Field.build`` for scalar fields (core/field.py:364-384, 616-740)."""
    spec = build_spectrum(spectrum, prec)
    u = prec.c(u)
    dx = np.atleast_1d(prec.r(dx))
    # utils/shapes.py:79-99 (_broadcast_dx_to_grid)
    if dx.shape == (1,):
        dxw = np.repeat(dx.reshape(1, 1), 2, axis=1).repeat(spec.size, axis=0)
    elif dx.ndim == 1:
        assert dx.shape[0] == spec.size, "Number of wavelengths does not match"
        dxw = np.repeat(dx[:, None], 2, axis=1)
    else:
        assert dx.shape == (spec.size, 2)
        dxw = dx
    if spec.mono:
        assert u.ndim >= 2
        return OField(u, dxw.reshape(2).astype(prec.real), spec, prec.r([0.0, 0.0]), prec)
    assert u.shape[-1] == spec.size
    return OField(u, dxw.astype(prec.real), spec, prec.r(np.zeros((spec.size, 2))), prec)


def field_empty(shape, dx, spectrum, prec: Prec = FP64) -> OField:
    """``Field.empty`` (core/field.py:386-407), scalar only."""
    spec = build_spectrum(spectrum, prec)
    if spec.mono:
        u = np.zeros(shape, dtype=prec.cplx)
    else:
        u = np.zeros((*shape, spec.size), dtype=prec.cplx)
    return field_build(u, dx, spec, prec)


def pad(field: OField, pad_width, cval=0.0) -> OField:
    """``pad`` (core/field.py:534-549)."""
    if isinstance(pad_width, (int, np.integer)):
        pad_width = (int(pad_width), int(pad_width))
    nd = field.u.ndim
    sd = [nd + d for d in field.spatial_dims]
    pw = [(0, 0)] * nd
    pw[sd[0]] = (pad_width[0], pad_width[0])
    pw[sd[1]] = (pad_width[1], pad_width[1])
    return field.replace(u=np.pad(field.u, pw, constant_values=cval))


def crop(field: OField, crop_width) -> OField:
    """``crop`` (core/field.py:552-570)."""
    if isinstance(crop_width, (int, np.integer)):
        crop_width = (int(crop_width), int(crop_width))
    nd = field.u.ndim
    sd = [nd + d for d in field.spatial_dims]
    sl = [slice(None)] * nd
    sl[sd[0]] = slice(crop_width[0], field.u.shape[sd[0]] - crop_width[0])
    sl[sd[1]] = slice(crop_width[1], field.u.shape[sd[1]] - crop_width[1])
    return field.replace(u=field.u[tuple(sl)])


def shift_grid(field: OField, shift_yx) -> OField:
    """``shift_grid`` (core/field.py:573-585)."""
    s = np.atleast_1d(field.prec.r(shift_yx))
    if s.size < 2:
        s = np.array([s[0], s[0]], dtype=field.prec.real)
    return field.replace(origin=np.zeros_like(field.origin) + s)


def l2_sq_norm(a, axis=-1):
    """``l2_sq_norm`` (utils/utils.py:138-140)."""
    return np.sum(a**2, axis=axis)


def _innermost_batch(x, field: OField):
    """``_broadcast_1d_to_innermost_batch`` (utils/shapes.py:52-58)."""
    x = np.atleast_1d(x)
    return x.reshape((x.size,) + (1,) * abs(field.spatial_dims[0]))


# ---------------------------------------------------------------------------
# propagators  (functional/propagation.py)
# ---------------------------------------------------------------------------


def compute_transfer_propagator(field: OField, z, n, kykx=(0.0, 0.0)):
    """Fresnel transfer kernel (functional/propagation.py:466-496)."""
    p = field.prec
    z = p.r(z)
    kykx = p.r(kykx)
    if z.size > 1:
        z = _innermost_batch(z, field)
    # -jnp.pi is a weak python float: (((-pi * lam) / n) * z) * |f - kykx|^2
    phase = (((p.real(-np.pi) * field.broadcasted_wavelength) / p.real(n)) * z) * l2_sq_norm(
        field.f_grid - kykx
    )
    H = np.exp(p.cplx(1j) * phase.astype(p.real)).astype(p.cplx)
    return np.fft.ifftshift(H, axes=field.spatial_dims)


def compute_asm_propagator(
    field: OField,
    z,
    n,
    kykx=(0.0, 0.0),
    bandlimit: bool = False,
    shift_yx=(0.0, 0.0),
    remove_evanescent: bool = False,
):
    """Angular-spectrum kernel (functional/propagation.py:499-580)."""
    p = field.prec
    z = p.r(z)
    kykx = p.r(kykx)
    shift_yx = p.r(shift_yx)
    if z.size > 1:
        z = _innermost_batch(z, field)
    lam = field.broadcasted_wavelength
    fg = field.f_grid
    kernel = p.real(1) - (lam / p.real(n)) ** 2 * l2_sq_norm(fg - kykx)
    kernel = kernel.astype(p.real)
    if remove_evanescent:
        delay = np.sqrt(np.maximum(kernel, p.real(0))).astype(p.real)
    else:
        delay = np.sqrt(kernel.astype(p.cplx))
    out_shift = (p.real(2 * np.pi) * np.sum(fg * shift_yx, axis=-1)).astype(p.real)
    A = (np.abs(z) * p.real(n) / lam).astype(p.real)
    phase = (p.real(2 * np.pi) * A) * delay + out_shift
    e = np.exp(p.cplx(1j) * phase.astype(p.cplx)).astype(p.cplx)
    kernel_field = np.where(z >= 0, e, np.conj(e))
    if bandlimit:
        # Matsushima 2010, Table 1 (functional/propagation.py:557-579), literal
        # broadcasting: valid for monochromatic fields and scalar z.
        df = field.df
        ext = field.extent
        k_limit_p = ((shift_yx + 1 / (2 * df)) ** (-2) * z**2 + 1) ** (-0.5) / lam
        k_limit_n = ((shift_yx - 1 / (2 * df)) ** (-2) * z**2 + 1) ** (-0.5) / lam
        k0 = 0.5 * (np.sign(shift_yx + ext) * k_limit_p + np.sign(shift_yx - ext) * k_limit_n)
        k_width = np.sign(shift_yx + ext) * k_limit_p - np.sign(shift_yx - ext) * k_limit_n
        k_max = k_width / 2
        Hyx = np.abs(fg - k0) <= k_max
        kernel_field = kernel_field * (Hyx[..., 0] * Hyx[..., 1])
    return np.fft.ifftshift(kernel_field.astype(p.cplx), axes=field.spatial_dims)


def kernel_propagate(
    field: OField,
    propagator,
    absorbing_boundary=None,
    absorbing_boundary_width: float = 0.65,
    output_dx=None,
    output_shape=None,
    shift_yx=(0.0, 0.0),
    use_czt: bool = False,
) -> OField:
    """Fourier-multiplier propagation (functional/propagation.py:355-463).

    The absorbing boundary of the reference is applied to the *input* field
    object and then discarded by ``field.replace(u=u)`` (lines 460-463), so it
    has no effect on the output; this restatement keeps that behaviour.
    """
    p = field.prec
    axes = field.spatial_dims
    shift_yx = p.r(shift_yx)
    if output_dx is None and output_shape is None and not use_czt:
        u = _ifft2(_fft2(field.u, axes) * propagator, axes).astype(p.cplx)
        field = shift_grid(field, shift_yx)
        return field.replace(u=u)
    if output_shape is None:
        output_shape = field.spatial_shape
    if output_dx is None:
        output_dx = field.dx
    in_u = field.u
    in_df = field.df
    in_fgrid = field.f_grid
    in_extent = np.squeeze(field.extent)
    field = shift_grid(field, shift_yx)
    out = _empty_like(field, output_shape, output_dx)
    alpha = out.dx / in_df
    u = np.fft.fftshift(
        propagator * _fft2(np.fft.ifftshift(in_u, axes=axes), axes), axes=axes
    ).astype(p.cplx)
    if use_czt:
        (y_min, y_max), (x_min, x_max) = spatial_limits(out)
        lo = [y_min, x_min]
        hi = [y_max, x_max]
        T = np.atleast_1d(in_extent)
        for d in range(2):
            m = output_shape[d]
            a = np.exp(p.cplx(-1j) * p.real(2 * np.pi) / T[d] * p.real(lo[d]))
            w = np.exp(p.cplx(1j) * (p.real(2 * np.pi) / T[d]) * p.real(hi[d] - lo[d]) / p.real(m - 1))
            u = czt(u, m, a, w, axis=axes[d], prec=p)
            N = (m - 1) // 2
            u = np.moveaxis(u, axes[d], -1)
            C = w ** (-N * np.arange(m, dtype=p.real)) * (a**N)
            u = (u * C.astype(p.cplx)).astype(p.cplx)
            u = np.moveaxis(u, -1, axes[d])
        u = (u * np.prod(p.real(1) / alpha)).astype(p.cplx)
    else:
        # Yu et al. rescaled convolution (functional/propagation.py:445-458)
        from scipy.signal import fftconvolve

        wn = alpha * in_fgrid
        f = np.prod(np.exp(p.cplx(-1j) * p.real(np.pi) / alpha * wn**2), axis=-1)
        B = u * np.prod((p.real(1) / alpha) * np.exp(p.cplx(1j) * p.real(np.pi) / alpha * wn**2), axis=-1)
        mod = np.prod(out.dx * np.exp(p.cplx(1j) * p.real(np.pi) / alpha * out.grid**2), axis=-1)
        u = (mod * fftconvolve(B, f, mode="same", axes=axes)).astype(p.cplx)
    return out.replace(u=u)


def _empty_like(field: OField, shape, dx) -> OField:
    """``Field.empty_like`` (core/field.py:316-362)."""
    dx = field.prec.r(dx)
    assert dx.ndim == field.dx.ndim
    sh = list(field.u.shape)
    d = field.spatial_dims
    sh[d[0]] = shape[0]
    sh[d[1]] = shape[1]
    return field.replace(u=np.zeros(sh, dtype=field.prec.cplx), dx=dx)


def spatial_limits(field: OField):
    """``Field.spatial_limits`` (core/field.py:221-229)."""
    g = field.grid
    return (float(g[..., 0].min()), float(g[..., 0].max())), (
        float(g[..., 1].min()),
        float(g[..., 1].max()),
    )


def transfer_propagate(
    field: OField,
    z,
    n,
    pad_width,
    cval=0.0,
    absorbing_boundary=None,
    absorbing_boundary_width=0.65,
    kykx=(0.0, 0.0),
    shift_yx=(0.0, 0.0),
    output_dx=None,
    output_shape=None,
    use_czt=True,
    mode="full",
) -> OField:
    """Fresnel transfer propagation (functional/propagation.py:168-252)."""
    field = pad(field, pad_width, cval)
    if output_dx is None and output_shape is None:
        use_czt = False
    z = np.atleast_1d(field.prec.r(z))
    H = compute_transfer_propagator(field, z, n, kykx)
    field = kernel_propagate(
        field, H, absorbing_boundary, absorbing_boundary_width, output_dx, output_shape, shift_yx, use_czt
    )
    if mode == "same":
        field = crop(field, pad_width)
    return field


def asm_propagate(
    field: OField,
    z,
    n,
    pad_width,
    cval=0.0,
    absorbing_boundary=None,
    absorbing_boundary_width=0.65,
    kykx=(0.0, 0.0),
    remove_evanescent=False,
    bandlimit=False,
    shift_yx=(0.0, 0.0),
    output_dx=None,
    output_shape=None,
    use_czt=True,
    mode="full",
) -> OField:
    """Angular-spectrum / exact propagation (functional/propagation.py:255-352)."""
    field = pad(field, pad_width, cval)
    if output_dx is None and output_shape is None:
        use_czt = False
    H = compute_asm_propagator(
        field,
        z,
        n,
        kykx,
        bandlimit,
        shift_yx if not use_czt else (0.0, 0.0),
        remove_evanescent=remove_evanescent,
    )
    field = kernel_propagate(
        field, H, absorbing_boundary, absorbing_boundary_width, output_dx, output_shape, shift_yx, use_czt
    )
    if mode == "same":
        field = crop(field, pad_width)
    return field


def transform_propagate(
    field: OField, z, n, pad_width, cval=0.0, skip_initial_phase=False, skip_final_phase=False
) -> OField:
    """Single-FFT Fresnel propagation (functional/propagation.py:34-82)."""
    p = field.prec
    field = pad(field, pad_width, cval)
    L_sq = field.broadcasted_wavelength * p.real(z) / p.real(n)
    if not skip_initial_phase:
        ph = (p.real(np.pi) / L_sq) * l2_sq_norm(field.grid)
        field = field.replace(u=(field.u * np.exp(p.cplx(1j) * ph)).astype(p.cplx))
    field = optical_fft(field, z, n)
    field = field.replace(u=(p.cplx(1j) * field.u).astype(p.cplx))
    if not skip_final_phase:
        ph = (p.real(np.pi) / L_sq) * l2_sq_norm(field.grid)
        field = field.replace(u=(field.u * np.exp(p.cplx(1j) * ph)).astype(p.cplx))
    return crop(field, pad_width)


def compute_sas_precompensation(field: OField, z, n):
    """SAS precompensation (functional/propagation.py:85-103)."""
    p = field.prec
    lam = field.broadcasted_wavelength
    kz = p.real(2) * p.real(z) * p.real(np.pi) * p.real(n) / lam
    s = lam * field.f_grid / p.real(n)
    s_sq = s**2
    L = 2 * field.extent
    t = L / 2 / np.abs(p.real(z)) + np.abs(s)
    W = np.prod((s_sq * (2 + 1 / t**2) <= 1), axis=-1)
    H_AS = np.sqrt(np.maximum(0, 1 - np.sum(s_sq, axis=-1)))
    H_Fr = 1 - np.sum(s_sq, axis=-1) / 2
    dH = W * np.exp(p.cplx(1j) * kz * (H_AS - H_Fr))
    return np.fft.ifftshift(dH.astype(p.cplx), axes=field.spatial_dims)


def transform_propagate_sas(field: OField, z, n, cval=0.0, skip_initial_phase=False, skip_final_phase=False):
    """Scalable ASM (functional/propagation.py:106-165)."""
    sz = np.array(field.spatial_shape)
    pw = tuple(int(v) for v in sz // 2)
    field = pad(field, pw, cval)
    if z >= 0:
        dH = compute_sas_precompensation(field, z, n)
        f2 = kernel_propagate(field, dH)
        f2 = transform_propagate(f2, z, n, 0, 0, skip_initial_phase, skip_final_phase)
    else:
        f2 = transform_propagate(field, z, n, 0, 0, skip_initial_phase, skip_final_phase)
        dH = compute_sas_precompensation(f2, z, n)
        f2 = kernel_propagate(f2, dH)
    field = field.replace(u=f2.u, dx=f2.dx)
    return crop(field, pw)


def compute_padding_transfer(height, wavelength, dx, z):
    """functional/propagation.py:608-630 (identical to the transform rule)."""
    D = height * dx
    Nf = np.max((D / 2) ** 2 / (wavelength * z))
    M = height
    Q = 2 * np.maximum(1.0, M / (4 * Nf))
    N = (np.ceil((Q * M) / 2) * 2).astype(int)
    return int(N - M)


compute_padding_transform = compute_padding_transfer  # functional/propagation.py:583-605


def compute_padding_exact(height, wavelength, dx, z):
    """functional/propagation.py:633-656."""
    D = height * dx
    Nf = np.max((D / 2) ** 2 / (wavelength * z))
    M = height
    Q = 2 * np.maximum(1.0, M / (4 * Nf))
    scale = np.max((wavelength / (2 * dx)))
    Q = Q / np.sqrt(1 - scale**2)
    N = (np.ceil((Q * M) / 2) * 2).astype(int)
    return int(N - M)


# ---------------------------------------------------------------------------
# lenses / optical FFT  (functional/convenience.py, functional/lenses.py)
# ---------------------------------------------------------------------------


def optical_fft(field: OField, z, n) -> OField:
    """Centred, scaled lens FFT (functional/convenience.py:9-59, utils/fft.py:8-20)."""
    p = field.prec
    z = p.real(z)
    L_sq = (field.broadcasted_wavelength * z / p.real(n)).astype(p.real)
    if field.spectrum.size > 1:
        _L = np.squeeze(L_sq).reshape(-1, *([1] * (field.df.ndim - 1)))
        du = field.df * np.abs(_L)
    else:
        du = field.df * np.abs(L_sq)
    axes = field.spatial_dims
    if z >= 0:
        norm = p.cplx(-1j) * np.prod(field.dx, axis=-1) / L_sq
        inp = norm * field.u
    else:
        norm = (
            p.cplx(-1j)
            * (L_sq / np.prod(du, axis=-1))
            / np.prod(np.array(field.spatial_shape, dtype=p.real))
        )
        inp = norm * np.conj(field.u)
    out = np.fft.fftshift(_fft2(np.fft.ifftshift(inp.astype(p.cplx), axes=axes), axes), axes=axes)
    if z < 0:
        out = np.conj(out)
    return field.replace(u=out.astype(p.cplx), dx=du.astype(p.real))


def circular_pupil(field: OField, w) -> OField:
    """functional/pupils.py:17-23."""
    p = field.prec
    r = (field.spectrum.central_wavelength / field.broadcasted_wavelength) * p.real(w) / p.real(2)
    mask = l2_sq_norm(field.grid) <= r**2
    return field.replace(u=(field.u * mask).astype(p.cplx))


def square_pupil(field: OField, w) -> OField:
    """functional/pupils.py:26-31."""
    p = field.prec
    half = (field.spectrum.central_wavelength / field.broadcasted_wavelength) * p.real(w) / p.real(2)
    mask = np.max(np.abs(field.grid), axis=-1) <= half
    return field.replace(u=(field.u * mask).astype(p.cplx))


def ff_lens(field: OField, f, n, NA=None, inverse=False) -> OField:
    """functional/lenses.py:64-95."""
    if NA is not None:
        field = circular_pupil(field, 2 * f * NA / n)
    if inverse:
        f = -f
    return optical_fft(field, f, n)


def thin_lens(field: OField, f, n, NA=None) -> OField:
    """functional/lenses.py:37-61."""
    p = field.prec
    L = np.sqrt(field.broadcasted_wavelength * p.real(f) / p.real(n))
    phase = -p.real(np.pi) * l2_sq_norm(field.grid) / L**2
    if NA is not None:
        field = circular_pupil(field, 2 * f * NA / n)
    return field.replace(u=(field.u * np.exp(p.cplx(1j) * phase)).astype(p.cplx))


def df_lens(field: OField, d, f, n, NA=None, inverse=False) -> OField:
    """functional/lenses.py:159-198 (inverse branch kept as written there)."""
    p = field.prec
    if NA is not None:
        field = circular_pupil(field, 2 * f * NA / n)
    if inverse:
        f = -d
        d = -f
    field = optical_fft(field, f, n)
    L = np.sqrt((field.broadcasted_wavelength * p.real(f) / p.real(n)).astype(p.cplx))
    phase = p.real(np.pi) * (1 - d / f) * l2_sq_norm(field.grid) / np.abs(L) ** 2
    return field.replace(u=(field.u * np.exp(p.cplx(1j) * phase)).astype(p.cplx))


# ---------------------------------------------------------------------------
# sources / masks / samples
# ---------------------------------------------------------------------------


def objective_point_source(shape, dx, spectrum, z, f, n, NA, power=1.0, amplitude=1.0,
                           offset=(0.0, 0.0), prec: Prec = FP64) -> OField:
    """Defocused point source behind an objective (functional/sources.py:122-209)."""
    p = prec
    field = field_empty(shape, dx, spectrum, p)
    amplitude = np.atleast_1d(p.r(amplitude))
    z = np.squeeze(np.atleast_1d(p.r(z)))
    if z.size > 1:
        z = _innermost_batch(z, field)
        field = field.replace(u=field.u[None])
    offset = np.atleast_1d(p.r(offset))
    lam = field.broadcasted_wavelength
    L = np.sqrt(lam * p.real(f) / p.real(n))
    phase = -p.real(np.pi) * (z / p.real(f)) * l2_sq_norm(field.grid - offset) / L**2
    u = amplitude * p.cplx(-1j) / L**2 * np.exp(p.cplx(1j) * phase)
    u = np.broadcast_to(u, np.broadcast_shapes(u.shape, field.u.shape)).astype(p.cplx)
    field = field.replace(u=u)
    D = 2 * f * NA / n
    field = circular_pupil(field, D)
    if power is not None:
        field = field.replace(u=(field.u * np.sqrt(p.real(power) / field.power)).astype(p.cplx))
    return field


def plane_wave(shape, dx, spectrum, power=1.0, amplitude=1.0, kykx=(0.0, 0.0), pupil=None,
               prec: Prec = FP64) -> OField:
    """functional/sources.py:212-293 (scalar fields)."""
    p = prec
    field = field_empty(shape, dx, spectrum, p)
    amplitude = np.atleast_1d(p.r(amplitude))
    kykx = np.atleast_1d(p.r(kykx))
    u = amplitude * np.exp(p.cplx(1j) * np.sum(kykx * field.grid, axis=-1))
    field = field.replace(u=(u * np.ones_like(field.u)).astype(p.cplx))
    if pupil is not None:
        field = pupil(field)
    if power is not None:
        field = field.replace(u=(field.u * np.sqrt(p.real(power) / field.power)).astype(p.cplx))
    return field


def phase_change(field: OField, phase, spectrally_modulate=True) -> OField:
    """functional/phase_masks.py:29-68, 105-124."""
    p = field.prec
    phase = p.r(phase)
    if phase.ndim != field.u.ndim:
        phase = phase.reshape(phase.shape + (1,) * (abs(field.spatial_dims[0]) - 2))
    if spectrally_modulate:
        phase = phase * field.spectrum.spectral_modulation
    return field.replace(u=(field.u * np.exp(p.cplx(1j) * phase)).astype(p.cplx))


def thin_sample(field: OField, absorption, dn, thickness) -> OField:
    """functional/samples.py:85-134."""
    p = field.prec
    ex = abs(field.spatial_dims[0]) - 2
    absorption = p.r(absorption).reshape(np.shape(absorption) + (1,) * ex)
    dn = p.r(dn).reshape(np.shape(dn) + (1,) * ex)
    # 1j * 2 * jnp.pi is folded by Python into one complex constant
    sample = np.exp(
        p.cplx(2j * np.pi) * (dn + p.cplx(1j) * absorption) * p.real(thickness)
        / field.broadcasted_wavelength
    )
    return field.replace(u=(field.u * sample).astype(p.cplx))


def center_pad(u, pad_width, cval=0):
    """utils/utils.py:15-22."""
    return np.pad(u, [(w, w) for w in pad_width], constant_values=cval)


def multislice_thick_sample(field: OField, absorption_stack, dn_stack, n, thickness_per_slice,
                            pad_width, NA=None, propagator=None, kykx=(0.0, 0.0),
                            reverse_propagate_distance=None, return_stack=False,
                            remove_evanescent=False, bandlimit=False) -> OField:
    """Thick-sample multislice (functional/samples.py:137-282)."""
    assert np.shape(absorption_stack) == np.shape(dn_stack)
    field = pad(field, pad_width)
    absorption_stack = center_pad(absorption_stack, (0, pad_width, pad_width))
    dn_stack = center_pad(dn_stack, (0, pad_width, pad_width))
    if propagator is None:
        propagator = compute_asm_propagator(field, thickness_per_slice, n, kykx,
                                            remove_evanescent=remove_evanescent, bandlimit=bandlimit)
    if return_stack:
        raise NotImplementedError("return_stack is not restated (samples.py:253-260)")
    u = field.u
    for i in range(dn_stack.shape[0]):
        fi = kernel_propagate(field.replace(u=u), propagator)
        fi = thin_sample(fi, absorption_stack[i], dn_stack[i], thickness_per_slice)
        u = fi.u
    field = field.replace(u=u)
    if reverse_propagate_distance is None:
        reverse_propagate_distance = thickness_per_slice * dn_stack.shape[0] / 2
    Hd = compute_asm_propagator(field, -reverse_propagate_distance, n, kykx=kykx)
    if NA is not None:
        mask = l2_sq_norm(field.f_grid) <= (NA / field.broadcasted_wavelength) ** 2
        mask = np.fft.ifftshift(mask, axes=field.spatial_dims)
        Hd = Hd * mask
    field = kernel_propagate(field, Hd)
    return crop(field, pad_width)


def polarized_multislice_thick_sample(u, dx, wavelength, potential_stack, n, thickness_per_slice, NA=1.0):
    """Birefringent multislice (functional/samples.py:444-546) of a
    monochromatic vector field ``u`` (y x 3, components z, y, x) through a
    (d y x 3 3) scattering potential, FP64: per slice
    u <- P_op(u) + H_op(V_i Q_op(u)) on the grid zero-padded to twice the size
    (padding after the data, crop of the first rows / columns)."""
    u = np.asarray(u, dtype=np.complex128)
    ny, nx = u.shape[:2]
    P, Q = 2 * ny, 2 * nx
    dy, dxx = (float(dx), float(dx)) if np.ndim(dx) == 0 else (float(dx[0]), float(dx[1]))
    # k grid of the field padded by N // 2 per side, ifftshifted (FFT order)
    ky = 2 * np.pi * np.fft.fftfreq(P, d=dy)
    kx = 2 * np.pi * np.fft.fftfreq(Q, d=dxx)
    KY, KX = np.meshgrid(ky, kx, indexing="ij")
    km = 2 * np.pi * n / wavelength
    kz = np.sqrt(np.maximum(0.0, km**2 - KY**2 - KX**2))
    k = np.stack([kz, KY, KX], axis=-1) / km
    Qm = np.eye(3) - k[..., :, None] * k[..., None, :]
    Qm = np.where(((KY**2 + KX**2) <= NA**2 * km**2)[..., None, None], Qm, 0.0)
    dz = thickness_per_slice
    with np.errstate(divide="ignore", invalid="ignore"):
        e = np.where(kz > 0, np.exp(1j * kz * dz), 0)
        h = np.where(kz > 0, -1j / 2 * np.exp(1j * kz * dz) / kz * dz, 0)

    def pad_op(v):
        return np.pad(v, [(0, ny), (0, nx), (0, 0)])

    def crop_op(v):
        return v[:ny, :nx]

    def fft(v):
        return np.fft.fft2(v, axes=(0, 1))

    def ifft(v):
        return np.fft.ifft2(v, axes=(0, 1))

    def matvec(M, v):
        return np.einsum("...ij,...j->...i", M, v)

    for V in np.asarray(potential_stack, dtype=np.float64):
        Qu = crop_op(ifft(matvec(Qm, fft(pad_op(u)))))
        s = matvec(V, Qu)
        u = crop_op(ifft(matvec(Qm, e[..., None] * fft(pad_op(u))))) + crop_op(
            ifft(matvec(Qm, h[..., None] * fft(pad_op(s)))))
    return u


def _fft_centred(x, axes, inverse=False):
    """``fft`` / ``ifft`` with shift=True (utils/fft.py:8-48)."""
    f = np.fft.ifftn if inverse else np.fft.fftn
    return np.fft.fftshift(f(np.fft.ifftshift(x, axes=axes), axes=axes), axes=axes)


def ray_transfer(field: OField, ABCD, n, magnification=1.0) -> OField:
    """Collins' integral through an ABCD system (functional/rays.py:102-154)."""
    A, B, D = ABCD[0][0], ABCD[0][1], ABCD[1][1]
    M = magnification
    lam = field.broadcasted_wavelength
    k = 2 * np.pi * n / lam
    input_phase = k / (2 * B) * (A - M) * l2_sq_norm(field.grid)
    transfer_phase = (np.pi * (lam / n) * B / M) * l2_sq_norm(field.f_grid)
    output_phase = k / (2 * B) * (D - 1 / M) * l2_sq_norm(field.grid / (M**2))
    axes = field.spatial_dims
    fft_input = field.u * np.exp(1j * input_phase)
    u = np.exp(1j * output_phase) * _fft_centred(_fft_centred(fft_input, axes) * np.exp(-1j * transfer_phase),
                                                 axes, inverse=True)
    return field.replace(u=u, dx=field.dx / M)


def fluor_phases(seed: int, sample: int, shape):
    """The counter-based phases of cx_fluorescent_multislice (no counterpart in
    the reference, which draws them with jax.random): splitmix64 of
    seed + (c + 1) * 0x9E3779B97F4A7C15 (mod 2^64), c = sample * size + index,
    top 24 bits as u in [0, 1), phase = float32(2 pi) * u in float32."""
    n = int(np.prod(shape))
    with np.errstate(over="ignore"):
        c = np.uint64(sample) * np.uint64(n) + np.arange(n, dtype=np.uint64)
        z = np.uint64(seed) + (c + np.uint64(1)) * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    u = (z >> np.uint64(40)).astype(np.float32) * np.float32(1.0 / 16777216.0)
    return (np.float32(2 * np.pi) * u).astype(np.float32).reshape(shape)


def fluorescent_multislice_thick_sample(field: OField, fluorescence_stack, dn_stack, n, thickness_per_slice,
                                        pad_width, phases, kykx=(0.0, 0.0), remove_evanescent=False,
                                        bandlimit=False):
    """Fluorescent thick sample (functional/samples.py:285-441) with the
    Monte-Carlo phases given, ``phases`` (num_samples, D, h, w): per sample the
    forward slices u <- ifft2(fft2(fl_i e^(i ph_i) + u e^(i 2 pi dn_i dz / lam)) Hf),
    then U = fft2(u) and I[D-1-i] += |crop(ifft2(U Hb^(i+1)))|^2; the field
    (U Hb^D after a sample) carries into the next sample as in the reference's
    fori_loop; I / num_samples."""
    fluorescence_stack = np.asarray(fluorescence_stack)
    dn_stack = np.asarray(dn_stack)
    assert fluorescence_stack.shape == dn_stack.shape
    phases = np.asarray(phases)
    S, D = phases.shape[0], dn_stack.shape[0]
    original_shape = field.spatial_shape
    axes = field.spatial_dims
    field = pad(field, pad_width)
    dn = center_pad(dn_stack, (0, pad_width, pad_width))
    Hf = compute_asm_propagator(field, thickness_per_slice, n, kykx, remove_evanescent=remove_evanescent,
                                bandlimit=bandlimit)
    Hb = compute_asm_propagator(field, -thickness_per_slice, n, kykx, remove_evanescent=remove_evanescent,
                                bandlimit=bandlimit)
    lam = field.broadcasted_wavelength
    intensity = np.zeros((D,) + tuple(original_shape))
    u = field.u
    for s in range(S):
        fl = center_pad(fluorescence_stack * np.exp(1j * phases[s]), (0, pad_width, pad_width))
        for i in range(D):
            u = u * np.exp(1j * 2 * np.pi * dn[i] * thickness_per_slice / lam)
            u = np.fft.ifftn(np.fft.fftn(fl[i] + u, axes=axes) * Hf, axes=axes)
        u = np.fft.fftn(u, axes=axes)
        for i in range(D):
            u = u * Hb
            fi = field.replace(u=np.fft.ifftn(u, axes=axes))
            intensity[D - 1 - i] += crop(fi, pad_width).intensity
    return intensity / S


def multislice_loss_and_grad(u0, dn_stack, absorption_stack, target, n, dz, wavelength, dx, NA=None,
                             reverse_propagate_distance=None):
    """FP64 reference for the differentiable multislice benchmark.

    Loss ``L = sum((|u_out|^2 - target)^2)`` with ``u_out`` the mono scalar
    field after ``multislice_thick_sample`` (pad 0).  Returns ``(L, dL/d dn,
    dL/d absorption, u_out)``, obtained by reverse-mode differentiation of the
    forward recursion ``u_{i+1} = t_i * P(u_i)`` written out by hand (the
    reference itself differentiates the same recursion with ``jax.grad``,
    functional/samples.py:236-264).
    """
    spec = build_spectrum(float(wavelength), FP64)
    field = field_build(np.asarray(u0, np.complex128), dx, spec, FP64)
    H = compute_asm_propagator(field, dz, n)
    D = dn_stack.shape[0]
    k = 2 * np.pi / wavelength
    us = [field.u]
    for i in range(D):
        v = _ifft2(_fft2(us[-1], (-2, -1)) * H, (-2, -1))
        t = np.exp(1j * k * dz * (dn_stack[i] + 1j * absorption_stack[i]))
        us.append(v * t)
    if reverse_propagate_distance is None:
        reverse_propagate_distance = dz * D / 2
    Hd = compute_asm_propagator(field, -reverse_propagate_distance, n)
    if NA is not None:
        mask = l2_sq_norm(field.f_grid) <= (NA / wavelength) ** 2
        Hd = Hd * np.fft.ifftshift(mask)
    u_out = _ifft2(_fft2(us[-1], (-2, -1)) * Hd, (-2, -1))
    I = np.abs(u_out) ** 2
    L = float(np.sum((I - target) ** 2))
    g = 4 * (I - target) * u_out
    g = _ifft2(_fft2(g, (-2, -1)) * np.conj(Hd), (-2, -1))
    gdn = np.zeros(dn_stack.shape)
    gab = np.zeros(dn_stack.shape)
    for i in range(D - 1, -1, -1):
        u1 = us[i + 1]
        w = g * np.conj(u1)
        gdn[i] = k * dz * np.imag(w)
        gab[i] = -k * dz * np.real(w)
        t = np.exp(1j * k * dz * (dn_stack[i] + 1j * absorption_stack[i]))
        g = _ifft2(_fft2(g * np.conj(t), (-2, -1)) * np.conj(H), (-2, -1))
    return L, gdn, gab, u_out


# ---------------------------------------------------------------------------
# chirp-Z transform  (utils/czt.py)
# ---------------------------------------------------------------------------


def czt(x, m, a, w, axis=-1, prec: Prec = FP64):
    """Bluestein chirp-Z transform along one axis (utils/czt.py:7-52)."""
    p = prec
    x = p.c(x)
    n = x.shape[axis]
    n_czt = m + n - 1
    k = np.arange(n_czt, dtype=p.real)
    a = p.cplx(a)
    w = p.cplx(w)
    wk2 = (w ** (k**2 / p.real(2))).astype(p.cplx)
    Awk2 = (a ** -k[:n] * wk2[:n]).astype(p.cplx)
    Fwk2 = np.fft.fft(p.cplx(1) / np.hstack((wk2[n - 1 : 0 : -1], wk2[:m])), n_czt).astype(p.cplx)
    wk2 = wk2[:m]
    x = np.moveaxis(x, axis, -1)
    y = np.fft.ifft(np.fft.fft(x * Awk2, n_czt, axis=-1) * Fwk2, axis=-1).astype(p.cplx)
    y = y[..., n - 1 : n + m - 1] * wk2
    return np.moveaxis(y.astype(p.cplx), -1, axis)


def cztn(x, m, a, w, axes=(-2, -1), prec: Prec = FP64):
    """utils/czt.py:55-80."""
    for d, ax in enumerate(axes):
        x = czt(x, m[d], a[d], w[d], axis=ax, prec=prec)
    return x


def zoomed_fft(x, k_start, k_end, output_shape, axes=(-2, -1), include_end=True, prec: Prec = FP64):
    """utils/czt.py:83-124."""
    renorm = tuple(m - 1 for m in output_shape) if include_end else tuple(output_shape)
    w = tuple(np.exp(1j * (k_end - k_start) / nn) for nn in renorm)
    a = np.exp(-1j * k_start)
    return cztn(x, output_shape, tuple(a for _ in output_shape), w, axes, prec)


def pupil_grid(shape, dx, origin=(0.0, 0.0)):
    """Spatial grid of a monochromatic field (core/field.py:23-33, 759-770):
    dx * (i - N/2) + origin, shape (y x 2), FP64."""
    ny, nx = shape
    dy, dxx = (float(dx), float(dx)) if np.ndim(dx) == 0 else (float(dx[0]), float(dx[1]))
    gy = (np.arange(ny) - ny / 2) * dy + origin[0]
    gx = (np.arange(nx) - nx / 2) * dxx + origin[1]
    GY, GX = np.meshgrid(gy, gx, indexing="ij")
    return np.stack([GY, GX], axis=-1)


def cartesian_to_spherical(u, grid, n, NA, f):
    """``cartesian_to_spherical`` (core/field.py:897-940): the pupil field of a
    vector field ``u`` (y x 3, components z, y, x) in the spherical basis of a
    lens of focal length f (Eq. 6 of arXiv:2502.03170), returned as (z, y, x)."""
    pupil_radius = f * NA / n
    radius_sq = np.sum(grid**2, axis=-1)
    mask = radius_sq <= pupil_radius**2
    sin_theta2 = radius_sq * mask / f**2
    cos_theta = np.sqrt(1 - sin_theta2)
    sin_theta = np.sqrt(sin_theta2)
    phi = np.arctan2(grid[..., 0], grid[..., 1])
    cos_phi, sin_phi = np.cos(phi), np.sin(phi)
    sin_2phi = 2 * sin_phi * cos_phi
    cos_2phi = cos_phi**2 - sin_phi**2
    fx, fy = u[..., 2], u[..., 1]
    e_x = ((cos_theta + 1.0) + (cos_theta - 1.0) * cos_2phi) * fx + (cos_theta - 1.0) * sin_2phi * fy
    e_y = ((cos_theta + 1.0) - (cos_theta - 1.0) * cos_2phi) * fy + (cos_theta - 1.0) * sin_2phi * fx
    e_z = -2.0 * sin_theta * (cos_phi * fx + sin_phi * fy)
    return np.stack([e_z, e_y, e_x], axis=-1) / 2


def high_na_ff_lens(u, dx, wavelength, f, n, NA, output_shape=None, output_dx=None, origin=(0.0, 0.0)):
    """``high_na_ff_lens`` (functional/lenses.py:98-156) of a monochromatic
    square field: ``u`` (y x) scalar or (y x 3) vectorial.  The defocus
    exp(i k sz f) / sz on the pupil's frequency grid, then a zoomed FFT over
    [-zoom pi, zoom pi] with the end point, zoom = 2 NA fov_out / ((N - 1)
    lambda).  Returns (u_out, output_dx)."""
    u = np.asarray(u, dtype=np.complex128)
    vectorial = u.ndim == 3
    shape = u.shape[:2]
    if vectorial:
        spherical_u = cartesian_to_spherical(u, pupil_grid(shape, dx, origin), n, NA, f)
    else:
        spherical_u = u
    if output_dx is None:
        output_dx = float(dx) if np.ndim(dx) == 0 else float(dx[0])
    if output_shape is None:
        output_shape = shape
    fov_out = output_shape[0] * output_dx
    zoom_factor = 2 * NA * fov_out / ((u.shape[1] - 1) * wavelength)
    fg = freq_grid(shape, np.broadcast_to(np.asarray(dx, np.float64), (2,)).reshape(1, 2), FP64, False)
    s_grid = fg * wavelength / n
    sz_sq = 1 - NA**2 * np.sum(s_grid**2, axis=-1)
    sz = np.sqrt(np.maximum(sz_sq, 0.0))
    k = 2 * np.pi * n / wavelength
    with np.errstate(divide="ignore", invalid="ignore"):
        defocus = np.where(sz != 0.0, np.exp(1j * k * sz * f) / sz, 0.0)
    if vectorial:
        defocus = defocus[..., None]
    axes = (0, 1)
    out = zoomed_fft(spherical_u * defocus, -zoom_factor * np.pi, zoom_factor * np.pi, tuple(output_shape),
                     axes=axes, include_end=True)
    return out, output_dx


# ---------------------------------------------------------------------------
# modified Born series  (experimental/modified_born_series/)
# ---------------------------------------------------------------------------

from scipy import constants as _const

MU0_C_1E6 = 1e-6 * _const.c * _const.mu_0  # experimental/modified_born_series/sample.py:79


def mbs_k_grid(shape, spacing):
    """``Sample.k_grid`` (experimental/modified_born_series/sample.py:46-58)."""
    ks = [np.fft.fftfreq(nn) for nn in shape]
    g = np.stack(np.meshgrid(*ks, indexing="ij"), axis=-1)
    return 2 * np.pi * g / spacing


def mbs_add_absorbing_bc(permittivity, spacing, axis, thickness, max_extinction=0.25, n_background=1.0):
    """experimental/modified_born_series/sample.py:88-124."""
    if not isinstance(axis, tuple):
        axis = (axis,)
    bw = int(thickness / spacing)
    bs = tuple((bw, bw) if i in axis else (0, 0) for i in range(3))
    ext = np.pad(np.zeros(permittivity.shape), bs, mode="linear_ramp", end_values=max_extinction)
    eps = (n_background + 1j * ext) ** 2
    perm = np.pad(permittivity, bs, mode="constant", constant_values=n_background**2)
    roi = tuple(slice(w, w + s) for (w, _), s in zip(bs, permittivity.shape))
    return perm + (eps - n_background**2), roi


def mbs_shift_and_scale(permittivity):
    """Shift/scale of experimental/modified_born_series/solver.py:10-39.

    The reference minimises ``max|eps - s|^2`` over complex ``s`` with
    optimistix NonlinearCG (rtol=atol=1e-3); the exact minimiser is the centre
    of the smallest circle enclosing the permittivity values in the complex
    plane, computed here exactly (Welzl) on the convex hull of the distinct
    values.  Returns ``(shift, 1/scale)`` with ``scale = 1.1j*radius``.
    """
    c, r = min_enclosing_circle(np.unique(np.asarray(permittivity).ravel()))
    scale = 1.1j * r
    return c, 1 / scale


def min_enclosing_circle(pts):
    pts = np.asarray(pts, dtype=np.complex128).ravel()
    if pts.size > 64:
        try:
            from scipy.spatial import ConvexHull

            P = np.stack([pts.real, pts.imag], 1)
            hull = ConvexHull(P)
            pts = pts[hull.vertices]
        except Exception:  # degenerate (collinear) point sets
            re = pts.real
            im = pts.imag
            idx = {int(np.argmin(re)), int(np.argmax(re)), int(np.argmin(im)), int(np.argmax(im))}
            pts = pts[sorted(idx)]
    pts = list(pts)
    rng = np.random.default_rng(0)
    rng.shuffle(pts)

    def circ2(a, b):
        c = (a + b) / 2
        return c, abs(a - c)

    def circ3(a, b, c):
        ax, ay, bx, by, cx, cy = a.real, a.imag, b.real, b.imag, c.real, c.imag
        d = 2 * (ax * (by - cy) + bx * (cy - ay) + cx * (ay - by))
        if abs(d) < 1e-300:
            cands = [circ2(a, b), circ2(a, c), circ2(b, c)]
            return max(cands, key=lambda t: t[1])
        ux = ((ax**2 + ay**2) * (by - cy) + (bx**2 + by**2) * (cy - ay) + (cx**2 + cy**2) * (ay - by)) / d
        uy = ((ax**2 + ay**2) * (cx - bx) + (bx**2 + by**2) * (ax - cx) + (cx**2 + cy**2) * (bx - ax)) / d
        ctr = complex(ux, uy)
        return ctr, abs(a - ctr)

    def inside(cr, p):
        return abs(p - cr[0]) <= cr[1] * (1 + 1e-12) + 1e-15

    cr = (pts[0], 0.0)
    for i in range(1, len(pts)):
        if inside(cr, pts[i]):
            continue
        cr = (pts[i], 0.0)
        for j in range(i):
            if inside(cr, pts[j]):
                continue
            cr = circ2(pts[i], pts[j])
            for k in range(j):
                if not inside(cr, pts[k]):
                    cr = circ3(pts[i], pts[j], pts[k])
    return cr


class MBSOperator:
    """``precondition`` (experimental/modified_born_series/solver.py:42-98), FP64."""

    def __init__(self, permittivity, spacing, k0, source_field, shift=None, scale=None):
        self.perm = np.asarray(permittivity, np.complex128)
        kg = mbs_k_grid(self.perm.shape, spacing) / k0
        self.kg = kg
        self.ksq = np.sum(kg**2, axis=-1, keepdims=True)
        if shift is None:
            shift, scale = mbs_shift_and_scale(self.perm)
        self.bias, self.scale = shift, scale
        self.kbsq = self.bias * self.scale + 1
        y = self.prec(np.asarray(source_field, np.complex128))
        self.num_scale = float(np.max(np.abs(y)))
        self.prec_y = y / self.num_scale

    def disc(self, x):
        return x * (self.scale * self.perm[..., None] - self.kbsq)

    def approx_inv(self, y):
        yf = _fftn(y, (0, 1, 2))
        proj = np.sum(self.kg * yf, axis=-1, keepdims=True)
        with np.errstate(invalid="ignore", divide="ignore"):
            ylong = np.where(self.ksq != 0, self.kg / self.ksq * proj, 0.0)
        ytr = yf - ylong
        yi = ytr / (self.kbsq - self.scale * self.ksq) + ylong / self.kbsq
        return _ifftn(yi, (0, 1, 2))

    def prec(self, y):
        return -self.disc(self.approx_inv(y * self.scale))

    def forward(self, x):
        return -self.disc(self.approx_inv(self.disc(x)) + x)

    def step(self, x):
        """One fixed-point update ``x <- prec_y - prec_forward(x) + x`` (solver.py:136-142)."""
        return self.prec_y - self.forward(x) + x


def mbs_solve(permittivity, spacing, k0, source_field, maxiter=1000, tol=1e-5, shift=None, scale=None):
    """Fixed-point MBS solve; stops when ||x_{k+1}-x_k|| / ||x_{k+1}|| < tol (FP64)."""
    op = MBSOperator(permittivity, spacing, k0, source_field, shift, scale)
    x = op.prec_y.copy()
    it = 0
    res = np.inf
    for it in range(1, maxiter + 1):
        xn = op.step(x)
        res = np.linalg.norm(xn - x) / max(np.linalg.norm(xn), 1e-300)
        x = xn
        if res < tol:
            break
    return x * op.num_scale, it, res, op


def mbs_bicgstab(op: "MBSOperator", x0, maxiter=1000, tol=1e-5):
    """BiCGStab on ``op.forward(x) = op.prec_y`` (solver.py:143-144, which calls
    jax.scipy.sparse.linalg.bicgstab), FP64: the published algorithm (van der
    Vorst 1992) with the stopping rule ||r|| <= tol ||b|| and the breakdown
    exits.  Returns (x, iterations, ||r|| / ||b||)."""
    b = op.prec_y
    vd = lambda a, c: np.vdot(a.reshape(-1), c.reshape(-1))
    x = np.asarray(x0, np.complex128).copy()
    r = b - op.forward(x)
    rhat = r.copy()
    p = r.copy()
    q = r.copy()
    rho = alpha = omega = 1.0 + 0j
    bs = float(np.real(vd(b, b)))
    thr2 = tol * tol * bs
    it = 0
    while float(np.real(vd(r, r))) > thr2 and it < maxiter:
        rho_new = vd(rhat, r)
        if rho_new == 0:
            break
        beta = rho_new / rho * alpha / omega
        p = r + beta * (p - omega * q)
        q = op.forward(p)
        alpha = rho_new / vd(rhat, q)
        s = r - alpha * q
        it += 1
        if float(np.real(vd(s, s))) < thr2:
            x = x + alpha * p
            r = s
            break
        t = op.forward(s)
        omega = vd(t, s) / vd(t, t)
        x = x + alpha * p + omega * s
        r = s - omega * t
        rho = rho_new
        if alpha == 0 or omega == 0:
            break
    return x, it, float(np.sqrt(np.real(vd(r, r)) / bs))


def mbs_source_field(current_density, k0):
    """``Source`` (experimental/modified_born_series/sample.py:75-85)."""
    return -1j / k0 * MU0_C_1E6 * np.asarray(current_density)


# ---------------------------------------------------------------------------
# incoherent imaging  (ops/ops.py, functional/sensors.py, systems/microscopes.py)
# ---------------------------------------------------------------------------


def next_order(val: int) -> int:
    """``next_order`` (utils/utils.py:11-12): the next power of two."""
    return int(2 ** np.ceil(np.log2(val)))


def fourier_convolution(image, kernel, axes=(0, 1), fast_fft_shape=True, mode="same"):
    """``fourier_convolution`` (ops/ops.py:9-86): rfftn/irfftn of real inputs at
    the (next power of two of the) summed shape, cropped to ``image``'s shape
    from offset (k - 1) // 2 for mode "same"."""
    image = np.asarray(image)
    kernel = np.asarray(kernel)
    axes = [a if a >= 0 else image.ndim + a for a in axes]
    padded = [image.shape[a] + kernel.shape[a] for a in axes]
    fast = [next_order(k) for k in padded] if fast_fft_shape else padded
    if np.iscomplexobj(image) or np.iscomplexobj(kernel):
        conv = np.fft.ifftn(np.fft.fftn(image, s=fast, axes=axes) * np.fft.fftn(kernel, s=fast, axes=axes),
                            s=fast, axes=axes)
    else:
        conv = np.fft.irfftn(np.fft.rfftn(image, s=fast, axes=axes) * np.fft.rfftn(kernel, s=fast, axes=axes),
                             s=fast, axes=axes)
    if mode == "same":
        sl = tuple(slice((k - 1) // 2, (k - 1) // 2 + i) if idx in axes else slice(i)
                   for idx, (i, k) in enumerate(zip(image.shape, kernel.shape)))
        conv = conv[sl]
    return conv


def basic_sensor_reduce(intensity, reduce_axis=None):
    """``basic_sensor`` (functional/sensors.py:14-92) without resampling or
    shot noise: the optional sum over ``reduce_axis``."""
    return np.sum(intensity, axis=reduce_axis) if reduce_axis is not None else intensity


def optical_4f_required_spacing(height, output_spacing, f_tube, n, wavelength):
    """``Optical4FSystemPSF.compute_required_spacing`` (systems/microscopes.py:357-365)."""
    return f_tube * np.asarray(wavelength, np.float64) / (n * height * output_spacing)


def microscope_image(sample, shape, spacing, f_tube, phase, f, n, NA, spectrum, z, reduce_axis=0,
                     prec: Prec = FP64):
    """``Microscope(Optical4FSystemPSF, BasicSensor(resampling_method=None))``
    called on ``sample`` (systems/microscopes.py:197-213, 271-297, 334-355):
    PSF intensity of the 4f system at every z, one plane-wise 2D Fourier
    convolution per z (axes (-2, -1)), the sensor's sum over ``reduce_axis``.
    padding_ratio = 0 and taper_width = 0 (the defaults)."""
    spec = build_spectrum(spectrum, prec)
    dx = optical_4f_required_spacing(shape[0], spacing, f_tube, n, spec.wavelength)
    dxw = dx if spec.wavelength.size > 1 else float(dx.reshape(-1)[0])
    fld = objective_point_source(shape, dxw, spectrum, z, f, n, NA, prec=prec)
    fld = ff_lens(phase_change(fld, phase), f_tube, n)
    psf = fld.intensity
    image = fourier_convolution(sample, psf, axes=(-2, -1))
    return basic_sensor_reduce(image, reduce_axis), psf


# ---------------------------------------------------------------------------
# misc helpers used by tests / baselines
# ---------------------------------------------------------------------------


def rel_l2(a, b) -> float:
    """Relative L2 error ``||a-b|| / ||b||`` in float64."""
    a = np.asarray(a, np.complex128)
    b = np.asarray(b, np.complex128)
    nb = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (nb if nb > 0 else 1.0))


def fresnel_square_aperture(x, z, w, wavelength, n):
    """Analytic Fresnel field of a square aperture (tests/test_propagate.py:17-33)."""
    from scipy.special import fresnel

    Nf = (w / 2) ** 2 / (wavelength / n * z)

    def I(xx):
        Smin, Cmin = fresnel(np.sqrt(2 * Nf) * (1 - 2 * xx / w))
        Splus, Cplus = fresnel(np.sqrt(2 * Nf) * (1 + 2 * xx / w))
        return 1 / np.sqrt(2) * (Cmin + Cplus) + 1j / np.sqrt(2) * (Smin + Splus)

    U = np.exp(1j * 2 * np.pi * z * n / wavelength) / 1j * I(x[..., 0]) * I(x[..., 1])
    return U / w
