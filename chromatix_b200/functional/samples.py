"""Thin and thick samples (functional/samples.py:85-282)."""

from __future__ import annotations

import numpy as np

from .. import _native as nat
from ..core.field import Field

__all__ = ["thin_sample"]


def thin_sample(field: Field, absorption, dn, thickness) -> Field:
    """``u * exp(1j 2 pi (dn + 1j absorption) thickness / lambda)``
    (functional/samples.py:85-134).  Inside ``multislice_thick_sample`` this
    product is fused into the slice kernel."""
    from .sources import materialize

    torch = nat.torch_mod()
    field = materialize(field)
    a = torch.as_tensor(np.asarray(absorption) if not isinstance(absorption, torch.Tensor) else absorption)
    d = torch.as_tensor(np.asarray(dn) if not isinstance(dn, torch.Tensor) else dn)
    if a.ndim != 2 or d.ndim != 2:
        raise AssertionError(f"Absorption and dn must have shape {field.spatial_shape}")
    a = a.to(device=field.device, dtype=torch.float64)
    d = d.to(device=field.device, dtype=torch.float64)
    lam = torch.as_tensor(field.spectrum.wavelength, device=field.device)
    if field.chromatic:
        a = a[..., None]
        d = d[..., None]
    else:
        lam = lam[0]
    arg = 2 * np.pi * thickness / lam
    t = torch.polar(torch.exp(-arg * a), arg * d).to(torch.complex64)
    return field.replace(u=field.u * t)
