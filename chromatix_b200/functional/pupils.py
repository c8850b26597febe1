"""Pupils (functional/pupils.py:17-67).

These masks are fused into the FFT loaders where they sit on the hot path
(``ff_lens``, ``objective_point_source``); the standalone functions below apply
them as device-side elementwise products for API completeness.
"""

from __future__ import annotations

import numpy as np

from .. import _native as nat
from ..core.field import Field

__all__ = ["circular_pupil", "square_pupil", "super_gaussian_pupil", "tukey_pupil"]


def _apply(field: Field, mask: np.ndarray) -> Field:
    from .sources import materialize

    torch = nat.torch_mod()
    field = materialize(field)
    m = torch.as_tensor(mask.astype(np.float32), device=field.device)
    return field.replace(u=field.u * m)


def _scale(field: Field):
    return field.spectrum.central_wavelength / field.broadcasted_wavelength


def circular_pupil(field: Field, w) -> Field:
    """|r|^2 <= ((lam0/lam) w / 2)^2 (functional/pupils.py:17-23)."""
    g = field._grid_np()
    return _apply(field, np.sum(g**2, axis=-1) <= (_scale(field) * w / 2) ** 2)


def square_pupil(field: Field, w) -> Field:
    """max(|y|, |x|) <= (lam0/lam) w / 2 (functional/pupils.py:26-31)."""
    g = field._grid_np()
    return _apply(field, np.max(np.abs(g), axis=-1) <= _scale(field) * w / 2)


def super_gaussian_pupil(field: Field, w, n=16) -> Field:
    """exp(-(|r| / w)^n) (functional/pupils.py:49-55)."""
    g = field._grid_np()
    return _apply(field, np.exp(-((np.sqrt(np.sum(g**2, axis=-1)) / w) ** n)))


def tukey_pupil(field: Field, w) -> Field:
    """Tukey window (functional/pupils.py:58-67)."""
    g = field._grid_np()
    ext = field.extent
    alpha = w / np.max(np.abs(ext), axis=-1)
    if field.chromatic:
        alpha = alpha.reshape(1, 1, -1)
    r = np.clip(np.sqrt(np.sum((g / ext) ** 2, axis=-1)), 0, 0.5)
    mask = np.where(r <= alpha / 2, 1.0, 0.5 * (1 + np.cos((2 * np.pi / (1 - alpha)) * (r - alpha / 2))))
    return _apply(field, mask)
