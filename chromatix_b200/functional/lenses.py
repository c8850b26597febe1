"""Lenses (functional/lenses.py): thin, front-focal-to-back-focal, d-to-f."""

from __future__ import annotations

import numpy as np

from .. import _native as nat
from ..core.field import Field
from .convenience import _dx_like, run_optfft
from .pupils import circular_pupil

__all__ = ["thin_lens", "ff_lens", "df_lens"]


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
