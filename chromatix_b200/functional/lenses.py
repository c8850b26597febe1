"""Lenses (functional/lenses.py): thin, front-focal-to-back-focal, d-to-f."""

from __future__ import annotations

import numpy as np

from .. import _native as nat
from ..core.field import Field
from .convenience import _dx_like, run_optfft
from .pupils import circular_pupil

__all__ = ["thin_lens", "ff_lens", "df_lens", "high_na_ff_lens"]


class cx_high_na_desc(nat.ctypes.Structure):
    _fields_ = ([(k, nat.c_int32) for k in ("n_fields", "ny", "nx", "my", "mx", "vectorial")] +
                [(k, nat.ctypes.c_double) for k in ("f", "n_medium", "NA", "wavelength", "dy", "dx", "origin_y",
                                                     "origin_x", "output_dx")])


def _high_na_lib():
    L = nat.lib()
    if not hasattr(L, "_cx_high_na_sig"):
        P = nat.ctypes.POINTER(cx_high_na_desc)
        L.cx_high_na_ff_lens_workspace_size.restype = nat.c_int32
        L.cx_high_na_ff_lens_workspace_size.argtypes = [P, nat.ctypes.POINTER(nat.c_size_t)]
        L.cx_high_na_ff_lens.restype = nat.c_int32
        L.cx_high_na_ff_lens.argtypes = [P, nat.c_void_p, nat.c_void_p, nat.c_void_p, nat.c_size_t, nat.c_void_p]
        L._cx_high_na_sig = True
    return L


def thin_lens(field: Field, f, n, NA=None) -> Field:
    """Quadratic lens phase exp(-i pi |r|^2 / (lam f / n)) (functional/lenses.py:37-61)."""
    from .sources import materialize

    torch = nat.torch_mod()
    field = materialize(field)
    L2 = field.broadcasted_wavelength * f / n
    g = field._grid_np()
    phase = -np.pi * np.sum(g**2, axis=-1) / L2
    if NA is not None:
        field = circular_pupil(field, 2 * f * NA / n)
    e = torch.as_tensor(np.exp(1j * phase).astype(np.complex64), device=field.device)
    return field.replace(u=field.u * e)


def ff_lens(field: Field, f, n, NA=None, inverse: bool = False, *, precision=None) -> Field:
    """Lens a focal length ``f`` after the field (functional/lenses.py:64-95):
    optional circular pupil of diameter 2 f NA / n, then ``optical_fft`` with
    ``f -> -f`` when ``inverse``.  A lazily built point source (optionally
    phase-masked) stays lazy so that ``.intensity`` runs the fused PSF kernel."""
    from .sources import LazySourceField, materialize

    if isinstance(field, LazySourceField) and field.stage in ("source", "phase") and not inverse and f > 0:
        return field.with_lens(float(f), float(n), NA)
    field = materialize(field)
    D = None if NA is None else 2 * f * NA / n
    if inverse:
        f = -f
    u, du = run_optfft(field, float(f), float(n), pupil_D=D, precision=precision)
    return field.replace(u=u, dx=_dx_like(field, du))


def df_lens(field: Field, d, f, n, NA=None, inverse: bool = False, *, precision=None) -> Field:
    """Lens a distance ``d`` after the field (functional/lenses.py:159-198):
    optical_fft by ``f`` then the residual quadratic phase
    pi (1 - d/f) |r|^2 / |L|^2 on the output grid, fused into the FFT store.
    The inverse branch keeps the reference's assignment order (f = -d; d = -f)."""
    from .sources import materialize

    field = materialize(field)
    D = None if NA is None else 2 * f * NA / n
    if inverse:
        f = -d
        d = -f
    f = float(f)
    L2 = np.abs(field.spectrum.wavelength * f / n)
    chirp = np.pi * (1 - d / f) / L2
    u, du = run_optfft(field, f, float(n), pupil_D=D, chirp_out=chirp, precision=precision)
    return field.replace(u=u, dx=_dx_like(field, du))


def high_na_ff_lens(field: Field, f, n, NA, output_shape=None, output_dx=None) -> Field:
    """High-NA lens a distance ``f`` after the field (functional/lenses.py:98-156):
    a vector field is first expressed in the lens's spherical basis
    (``cartesian_to_spherical``, core/field.py:897-940); then the defocus
    exp(i k sz f) / sz on the pupil's frequency grid and the zoomed FFT over
    [-zoom pi, zoom pi] onto ``output_shape`` with pixel pitch ``output_dx``,
    zoom = 2 NA output_shape[0] output_dx / ((nx - 1) lambda).  One native
    call (``cx_high_na_ff_lens``): an FP64 pupil pass and two fused chirp-Z
    passes.  Single wavelength, as in the reference; leading batch axes are
    independent fields."""
    from .sources import materialize

    torch = nat.torch_mod()
    field = materialize(field)
    nat.refuse_grad("high_na_ff_lens", field.u)
    if field.chromatic:
        raise NotImplementedError("high_na_ff_lens takes a single-wavelength field")
    nat.require_cuda(field.u, "field.u")
    ny, nx = field.spatial_shape
    if output_dx is None:
        output_dx = field.central_dx
    if output_shape is None:
        output_shape = (ny, nx)
    my, mx = int(output_shape[0]), int(output_shape[1])
    vect = bool(field.vectorial)
    batch = field.batch_shape
    n_fields = int(np.prod(batch)) if batch else 1
    dy, dxx = (float(v) for v in field.dx_wv[0])
    oy, ox = (float(v) for v in np.asarray(field.origin, dtype=np.float64).reshape(-1, 2)[0])
    d = cx_high_na_desc(n_fields=n_fields, ny=ny, nx=nx, my=my, mx=mx, vectorial=1 if vect else 0, f=float(f),
                        n_medium=float(n), NA=float(NA), wavelength=float(field.spectrum.wavelength[0]), dy=dy,
                        dx=dxx, origin_y=oy, origin_x=ox, output_dx=float(output_dx))
    L = _high_na_lib()
    wsb = nat.c_size_t(0)
    nat.check(L.cx_high_na_ff_lens_workspace_size(d, wsb))
    u = field.u.contiguous()
    ws = nat.workspace(wsb.value, u.device)
    out = torch.empty(tuple(batch) + (my, mx) + ((3,) if vect else ()), dtype=torch.complex64, device=u.device)
    nat.check(L.cx_high_na_ff_lens(d, nat.ptr(u), nat.ptr(out), nat.ptr(ws), wsb.value,
                                   nat.stream_handle(u.device)))
    new_dx = float(output_dx) * np.ones_like(np.asarray(field.dx, dtype=np.float64))
    return field.replace(u=out, dx=new_dx)
