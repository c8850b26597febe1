"""Field containers with the reference's scalar-field semantics.

``ScalarField`` (monochromatic, ``u`` of shape ``(... y x)``),
``ChromaticScalarField`` (``(... y x wv)``, wavelength innermost) and
``VectorField`` (monochromatic, ``(... y x 3)``, components z, y, x) mirror
core/field.py:49-811.  ``u`` is a CUDA ``complex64`` tensor; ``dx``,
``origin`` and the spectrum are float64 host arrays (they become per-plane
launch parameters).  Grids are returned as float32 device tensors, like the
reference's float32 jax arrays.
"""

from __future__ import annotations

import numpy as np

from .. import _native as nat
from .spectrum import MonoSpectrum, Spectrum


def _torch():
    return nat.torch_mod()


def grid(shape, spacing) -> np.ndarray:
    """``grid`` (core/field.py:23-33): dx * (i - N/2), shape (... y x 2)."""
    ny, nx = shape
    sp = np.asarray(spacing, dtype=np.float64)
    gy = np.arange(ny, dtype=np.float64) - ny / 2
    gx = np.arange(nx, dtype=np.float64) - nx / 2
    G = np.stack(np.meshgrid(gy, gx, indexing="ij"), axis=-1)
    return sp[..., None, None, :] * G


def freq_grid(shape, spacing) -> np.ndarray:
    """``freq_grid`` (core/field.py:36-46): fftshift(fftfreq(N)) / dx."""
    ny, nx = shape
    sp = np.asarray(spacing, dtype=np.float64)
    fy = np.fft.fftshift(np.fft.fftfreq(ny))
    fx = np.fft.fftshift(np.fft.fftfreq(nx))
    G = np.stack(np.meshgrid(fy, fx, indexing="ij"), axis=-1)
    return (1.0 / sp)[..., None, None, :] * G


def _broadcast_dx(dx, n_wv: int) -> np.ndarray:
    """``_broadcast_dx_to_grid`` (utils/shapes.py:79-99) -> (wv, 2)."""
    dx = np.atleast_1d(np.asarray(dx, dtype=np.float64))
    if dx.shape == (1,):
        out = np.repeat(dx.reshape(1, 1), 2, axis=1).repeat(n_wv, axis=0)
    elif dx.ndim == 1 and dx.shape[0] == 2 and n_wv == 1:
        out = dx.reshape(1, 2)
    elif dx.ndim == 1:
        if dx.shape[0] != n_wv:
            raise AssertionError("Number of wavelengths does not match")
        out = np.repeat(dx[:, None], 2, axis=1)
    elif dx.ndim == 2 and dx.shape == (n_wv, 2):
        out = dx
    else:
        raise ValueError(f"dx must be scalar or have shape (2,), (C,), or (C, 2); got {dx.shape}.")
    if np.any(out < 0):
        raise ValueError(f"dx must be larger than 0, got {out}.")
    return out


_INTENSITY_FN = None


def _intensity_launch(u, C: int, dens, out_shape):
    torch = _torch()
    out = torch.empty(out_shape, dtype=torch.float32, device=u.device)
    nat.check(nat.lib().cx_intensity(nat.ptr(u), out.numel(), C, nat.ptr(dens), nat.ptr(out),
                                     nat.stream_handle(u.device)))
    return out


def _intensity_fn():
    """autograd Function of the native intensity readout; the backward is
    ``cx_intensity_adjoint`` (g_u = 2 density g_I u)."""
    global _INTENSITY_FN
    if _INTENSITY_FN is None:
        torch = _torch()

        class _Intensity(torch.autograd.Function):
            @staticmethod
            def forward(ctx, u, C, dens, out_shape):
                ctx.C = C
                ctx.save_for_backward(u, dens)
                return _intensity_launch(u, C, dens, out_shape)

            @staticmethod
            def backward(ctx, g):
                u, dens = ctx.saved_tensors
                g = g.to(torch.float32).contiguous()
                gu = torch.empty_like(u)
                nat.check(nat.lib().cx_intensity_adjoint(nat.ptr(u), g.numel(), ctx.C, nat.ptr(dens), nat.ptr(g),
                                                         nat.ptr(gu), nat.stream_handle(u.device)))
                return gu, None, None, None

        _INTENSITY_FN = _Intensity
    return _INTENSITY_FN


def _intensity(u, C: int, density, out_shape):
    """sum_c density[c] |u[..., c]|^2 over C interleaved channels (native)."""
    torch = _torch()
    nat.require_cuda(u, "Field.u")
    u = u.to(torch.complex64).contiguous()
    dens = nat.upload(np.asarray(density, np.float64).reshape(-1), u.device)
    if nat.wants_grad(u):
        return _intensity_fn().apply(u, C, dens, tuple(out_shape))
    return _intensity_launch(u, C, dens, tuple(out_shape))


class Field:
    """Base of the scalar field containers (core/field.py:49-531)."""

    chromatic = False
    vectorial = False

    def __init__(self, u, dx, origin, spectrum: Spectrum):
        torch = _torch()
        if not isinstance(u, torch.Tensor):
            u = torch.as_tensor(np.asarray(u), dtype=torch.complex64)
        if u.dtype != torch.complex64:
            u = u.to(torch.complex64)
        self.u = u
        self.spectrum = spectrum
        self.dx = dx
        self.origin = origin

    # ---------------------------------------------------------------- layout
    @property
    def spatial_dims(self):
        if self.chromatic and self.vectorial:
            return (-4, -3)
        return (-3, -2) if (self.chromatic or self.vectorial) else (-2, -1)

    @property
    def shape(self):
        return tuple(self.u.shape)

    @property
    def spatial_shape(self):
        d = self.spatial_dims
        sh = self.shape
        return (sh[d[0]], sh[d[1]])

    @property
    def ndim(self) -> int:
        return len(self.shape)

    @property
    def batch_shape(self):
        return tuple(self.shape[: self.ndim + self.spatial_dims[0]])

    @property
    def batch_dims(self):
        return tuple(range(self.ndim + self.spatial_dims[0]))

    @property
    def num_batch_dims(self) -> int:
        return len(self.batch_dims)

    @property
    def n_wv(self) -> int:
        return self.spectrum.size if self.chromatic else 1

    @property
    def device(self):
        return self.u.device

    # ------------------------------------------------------------ spacing
    @property
    def dx_wv(self) -> np.ndarray:
        """Spacing as (wv, 2)."""
        return np.asarray(self.dx, dtype=np.float64).reshape(-1, 2)

    @property
    def extent(self) -> np.ndarray:
        return self.dx * np.asarray(self.spatial_shape, dtype=np.float64)

    @property
    def df(self) -> np.ndarray:
        return 1.0 / self.extent

    @property
    def surface_area(self) -> np.ndarray:
        return self.extent

    @property
    def wavelength(self) -> np.ndarray:
        return self.spectrum.wavelength

    @property
    def central_wavelength(self) -> float:
        return self.spectrum.central_wavelength

    @property
    def k(self) -> np.ndarray:
        return 2 * np.pi / self.wavelength

    @property
    def broadcasted_wavelength(self) -> np.ndarray:
        """``_broadcast_1d_to_channels`` (utils/shapes.py:26-43)."""
        wl = self.spectrum.wavelength
        if wl.size > 1:
            return wl.reshape(1, 1, wl.size)
        return wl.reshape(())

    @property
    def central_dx(self) -> float:
        return float(self.dx_wv[0, 0])

    # ------------------------------------------------------------ grids
    def _to_dev(self, a: np.ndarray):
        torch = _torch()
        return torch.as_tensor(a.astype(np.float32), device=self.device)

    def _grid_np(self) -> np.ndarray:
        g = grid(self.spatial_shape, self.dx_wv)  # (wv y x 2)
        org = np.asarray(self.origin, dtype=np.float64).reshape(-1, 2)
        if self.chromatic:
            return np.moveaxis(g, 0, 2) + org
        return g[0] + org[0]

    def _f_grid_np(self) -> np.ndarray:
        g = freq_grid(self.spatial_shape, self.dx_wv)
        return np.moveaxis(g, 0, 2) if self.chromatic else g[0]

    @property
    def grid(self):
        return self._to_dev(self._grid_np())

    @property
    def f_grid(self):
        return self._to_dev(self._f_grid_np())

    @property
    def k_grid(self):
        return self._to_dev(2 * np.pi * self._f_grid_np())

    @property
    def spatial_limits(self):
        g = self._grid_np()
        return (float(g[..., 0].min()), float(g[..., 0].max())), (float(g[..., 1].min()), float(g[..., 1].max()))

    # ------------------------------------------------------------ readouts
    @property
    def intensity(self):
        """|u|^2 (mono) or sum_wv density |u|^2 (core/field.py:656-665, 735-740),
        computed by the native readout kernel (differentiable: its adjoint is
        ``cx_intensity_adjoint``)."""
        u = self.u
        W = self.n_wv if self.chromatic else 1
        out_shape = u.shape[:-1] if self.chromatic else u.shape
        dens = np.asarray(self.spectrum.density, np.float64) if self.chromatic else np.ones(1)
        return _intensity(u, W, dens, out_shape)

    def intensity_to(self, out):
        """Write the intensity into ``out`` (a float32 tensor of the intensity's
        shape, on the device or in host memory) and return ``out``.  Host
        output is copied asynchronously when ``out`` is page-locked; it is
        valid once the current stream has been synchronised."""
        I = self.intensity
        if tuple(out.shape) != tuple(I.shape):
            raise ValueError(f"out has shape {tuple(out.shape)}, the intensity {tuple(I.shape)}")
        out.copy_(I, non_blocking=True)
        return out

    @property
    def power(self):
        """area * sum over (y, x) of the intensity (core/field.py:656-661, 728-733)."""
        torch = _torch()
        I = self.intensity
        pd = I.sum(dim=(-2, -1), dtype=torch.float64)
        area = torch.as_tensor(np.prod(self.dx_wv, axis=-1), device=I.device)
        if self.chromatic:
            return (area * pd[..., None, None, None]).to(torch.float32)
        return (area[0] * pd[..., None, None]).to(torch.float32)

    @property
    def phase(self):
        return _torch().angle(self.u)

    @property
    def amplitude(self):
        return self.u.abs()

    @property
    def conj(self):
        return self.replace(u=self.u.conj().resolve_conj())

    # ------------------------------------------------------------ pytree-ish
    def replace(self, **kw) -> "Field":
        new = object.__new__(type(self))
        new.__dict__.update(self.__dict__)
        for k, v in kw.items():
            setattr(new, k, v)
        return new

    @classmethod
    def build(cls, u, dx, spectrum) -> "Field":
        """``Field.build`` (core/field.py:364-384): (y x) scalar, (y x 3)
        vector, (y x wv) chromatic scalar; chromatic vector fields are not
        part of this build."""
        spec = Spectrum.build(spectrum)
        ndim = u.ndim
        if isinstance(spec, MonoSpectrum):
            if ndim == 3:
                return VectorField(u, dx, 0.0, spec)
            if ndim != 2:
                raise NotImplementedError(f"a monochromatic field has 2 (scalar) or 3 (vector) dimensions, got {ndim}")
            return ScalarField(u, dx, 0.0, spec)
        if ndim == 4:
            return ChromaticVectorField(u, dx, 0.0, spec)
        if ndim != 3:
            raise NotImplementedError(f"a chromatic field has 3 (scalar) or 4 (vector) dimensions, got {ndim}")
        return ChromaticScalarField(u, dx, 0.0, spec)

    @classmethod
    def empty(cls, shape, dx, spectrum, scalar: bool = True, device="cuda") -> "Field":
        """``Field.empty`` (core/field.py:386-407)."""
        return cls.zeros(shape, dx, spectrum, scalar, device)

    @classmethod
    def zeros(cls, shape, dx, spectrum, scalar: bool = True, device="cuda") -> "Field":
        """``Field.zeros`` (core/field.py:409-430), scalar fields."""
        if not scalar:
            raise NotImplementedError("vectorial fields are not part of this build")
        torch = _torch()
        spec = Spectrum.build(spectrum)
        if isinstance(spec, MonoSpectrum):
            u = torch.zeros(tuple(shape), dtype=torch.complex64, device=device)
        else:
            u = torch.zeros((*shape, spec.size), dtype=torch.complex64, device=device)
        return Field.build(u, dx, spec)

    @classmethod
    def empty_like(cls, field: "Field", shape=None, dx=None, origin=None, spectrum=None) -> "Field":
        """``Field.empty_like`` (core/field.py:316-362)."""
        torch = _torch()
        dx = field.dx if dx is None else np.asarray(dx, dtype=np.float64)
        if np.ndim(dx) != np.ndim(field.dx):
            raise AssertionError("New spacing must have same number of dimensions as old spacing")
        sh = list(field.shape)
        if shape is not None:
            sd = field.spatial_dims
            sh[sd[0]] = shape[0]
            sh[sd[1]] = shape[1]
        u = torch.zeros(tuple(sh), dtype=torch.complex64, device=field.device)
        return field.replace(u=u, dx=dx, origin=field.origin if origin is None else origin,
                             spectrum=field.spectrum if spectrum is None else spectrum)

    def expand_dims(self) -> "Field":
        return self.replace(u=self.u[None])

    unsqueeze = expand_dims

    def squeeze(self) -> "Field":
        u = self.u
        for d in reversed(self.batch_dims):
            if u.shape[d] == 1:
                u = u.squeeze(d)
        return self.replace(u=u)

    # ------------------------------------------------------------ arithmetic
    def _other(self, o):
        return o.u if isinstance(o, Field) else o

    def __add__(self, o):
        return self.replace(u=self.u + self._other(o))

    __radd__ = __add__

    def __sub__(self, o):
        return self.replace(u=self.u - self._other(o))

    def __rsub__(self, o):
        return self.replace(u=self._other(o) - self.u)

    def __mul__(self, o):
        return self.replace(u=self.u * self._other(o))

    __rmul__ = __mul__

    def __truediv__(self, o):
        return self.replace(u=self.u / self._other(o))

    def __rtruediv__(self, o):
        return self.replace(u=self._other(o) / self.u)

    def __neg__(self):
        return self.replace(u=-self.u)

    def __repr__(self):
        return (f"{type(self).__name__}(shape={self.shape}, dx={np.asarray(self.dx).tolist()}, "
                f"wavelength={self.spectrum.wavelength.tolist()})")


class ScalarField(Field):
    """Monochromatic scalar field, ``u`` of shape (... y x) (core/field.py:616-665)."""

    chromatic = False

    def __init__(self, u, dx, origin, spectrum):
        spec = spectrum if isinstance(spectrum, Spectrum) else MonoSpectrum(float(spectrum))
        super().__init__(u, _broadcast_dx(dx, 1).reshape(2),
                         np.broadcast_to(np.asarray(origin, dtype=np.float64), (2,)).copy(), spec)
        if self.u.ndim < 2:
            raise AssertionError(f"Expected 2-dimensional field, got shape {tuple(self.u.shape)}.")


class ChromaticScalarField(Field):
    """Chromatic scalar field, ``u`` of shape (... y x wv) (core/field.py:668-740)."""

    chromatic = True

    def __init__(self, u, dx, origin, spectrum: Spectrum):
        super().__init__(u, _broadcast_dx(dx, spectrum.size),
                         np.broadcast_to(np.asarray(origin, dtype=np.float64), (spectrum.size, 2)).copy(), spectrum)
        if self.u.ndim < 3:
            raise AssertionError(f"Expected 3-dimensional field, got shape {tuple(self.u.shape)}.")
        if self.u.shape[-1] != spectrum.size:
            raise AssertionError("Expected last dimension of u to be same as wavelengths.")


class VectorField(Field):
    """Monochromatic vector field, ``u`` of shape (... y x 3) with the
    components (z, y, x) innermost (core/field.py:743-811)."""

    chromatic = False
    vectorial = True

    def __init__(self, u, dx, origin, spectrum):
        spec = spectrum if isinstance(spectrum, Spectrum) else MonoSpectrum(float(spectrum))
        super().__init__(u, _broadcast_dx(dx, 1).reshape(2),
                         np.broadcast_to(np.asarray(origin, dtype=np.float64), (2,)).copy(), spec)
        if self.u.ndim < 3:
            raise AssertionError(f"Expected 3-dimensional field, got shape {tuple(self.u.shape)}.")
        if self.u.shape[-1] != 3:
            raise AssertionError(f"Expected last dimension of u to be 3, got {self.u.shape[-1]}")

    @property
    def intensity(self):
        """sum over the components of |u|^2 (core/field.py:808-811), by the
        native readout kernel."""
        return _intensity(self.u, 3, np.ones(3), self.u.shape[:-1])

    @property
    def power(self):
        """area * sum over (y, x) of the intensity (core/field.py:801-806)."""
        torch = _torch()
        pd = self.intensity.sum(dim=(-2, -1), dtype=torch.float64)
        return (float(np.prod(self.dx_wv[0])) * pd[..., None, None, None]).to(torch.float32)


class ChromaticVectorField(Field):
    """Chromatic vector field, ``u`` of shape (y x wv 3), components (z, y, x)
    innermost (core/field.py:813-894)."""

    chromatic = True
    vectorial = True

    def __init__(self, u, dx, origin, spectrum: Spectrum):
        super().__init__(u, _broadcast_dx(dx, spectrum.size),
                         np.broadcast_to(np.asarray(origin, dtype=np.float64), (spectrum.size, 2)).copy(), spectrum)
        if self.u.ndim != 4:
            raise AssertionError(f"Expected 4-dimensional field, got shape {tuple(self.u.shape)}.")
        if self.u.shape[-2] != spectrum.size:
            raise AssertionError("Expected last dimension of u to be same as wavelengths.")
        if self.u.shape[-1] != 3:
            raise AssertionError(f"Expected last dimension of u to be 3, got {self.u.shape[-1]}")

    @property
    def intensity(self):
        """sum over wavelengths (spectral density) and components of |u|^2
        (core/field.py:889-894), by the native readout kernel."""
        return _intensity(self.u, 3 * self.spectrum.size,
                          np.repeat(np.asarray(self.spectrum.density, np.float64), 3), self.u.shape[:-2])


def _channels(field: "Field") -> int:
    """Interleaved innermost values per pixel (wavelengths x vector components)."""
    return int(np.prod(field.u.shape[field.ndim + field.spatial_dims[1] + 1:]))


def _pad_native(u, batch: int, ny: int, nx: int, C: int, py: int, px: int, cval: complex):
    torch = _torch()
    d = nat.cx_ew_desc(n_batch=batch, ny=ny, nx=nx, n_wv=C, map_batched=0)
    out = torch.empty((batch, ny + 2 * py, nx + 2 * px, C), dtype=torch.complex64, device=u.device)
    nat.check(nat.lib().cx_pad(d, py, px, float(cval.real), float(cval.imag), nat.ptr(u.contiguous()), nat.ptr(out),
                               nat.stream_handle(u.device)))
    return out


_PAD_FN = None


def _pad_fn():
    """autograd Function of the native pad: the gradient is the crop."""
    global _PAD_FN
    if _PAD_FN is None:
        torch = _torch()

        class _Pad(torch.autograd.Function):
            @staticmethod
            def forward(ctx, u, dims, cval):
                batch, ny, nx, C, py, px = dims
                ctx.dims = dims
                ctx.in_shape = tuple(u.shape)
                return _pad_native(u, batch, ny, nx, C, py, px, cval)

            @staticmethod
            def backward(ctx, g):
                batch, ny, nx, C, py, px = ctx.dims
                g = g.reshape(batch, ny + 2 * py, nx + 2 * px, C)
                return g[:, py:py + ny, px:px + nx, :].reshape(ctx.in_shape), None, None

        _PAD_FN = _Pad
    return _PAD_FN


def pad(field: Field, pad_width, cval: float = 0.0) -> Field:
    """``pad`` (core/field.py:534-549): constant (``cval``) padding of y and x,
    one pass of the native pad kernel (``cx_pad``)."""
    if isinstance(pad_width, (int, np.integer)):
        pad_width = (int(pad_width), int(pad_width))
    py, px = int(pad_width[0]), int(pad_width[1])
    u = field.u
    nat.require_cuda(u, "Field.u")
    ny, nx = field.spatial_shape
    C = _channels(field)
    shape = tuple(u.shape)
    lead = shape[: field.ndim + field.spatial_dims[0]]
    batch = int(np.prod(lead)) if lead else 1
    cv = complex(cval)
    dims = (batch, ny, nx, C, py, px)
    if nat.wants_grad(u):
        out = _pad_fn().apply(u.to(_torch().complex64), dims, cv)
    else:
        out = _pad_native(u.to(_torch().complex64), batch, ny, nx, C, py, px, cv)
    inner = shape[field.ndim + field.spatial_dims[1] + 1:]
    return field.replace(u=out.reshape(lead + (ny + 2 * py, nx + 2 * px) + inner))


def crop(field: Field, crop_width) -> Field:
    """``crop`` (core/field.py:552-570)."""
    if isinstance(crop_width, (int, np.integer)):
        crop_width = (int(crop_width), int(crop_width))
    cy, cx = int(crop_width[0]), int(crop_width[1])
    d = field.spatial_dims
    ny, nx = field.spatial_shape
    idx = [slice(None)] * field.ndim
    idx[field.ndim + d[0]] = slice(cy, ny - cy)
    idx[field.ndim + d[1]] = slice(cx, nx - cx)
    return field.replace(u=field.u[tuple(idx)].contiguous())


def shift_grid(field: Field, shift_yx) -> Field:
    """``shift_grid`` (core/field.py:573-585): sets the origin."""
    s = np.atleast_1d(np.asarray(shift_yx, dtype=np.float64))
    if s.size < 2:
        s = np.array([s[0], s[0]])
    if s.size != 2:
        raise AssertionError("Shift must be an array of size (2,) in the order (y x)")
    return field.replace(origin=np.zeros_like(np.asarray(field.origin, dtype=np.float64)) + s)
