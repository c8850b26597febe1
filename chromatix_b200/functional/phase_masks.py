"""Phase masks (functional/phase_masks.py:29-68, 105-124)."""

from __future__ import annotations

import numpy as np

from .. import _native as nat
from ..core.field import Field

__all__ = ["phase_change", "spectrally_modulate_phase"]


def spectrally_modulate_phase(phase, spectrum):
    """phase * lambda0 / lambda (functional/phase_masks.py:105-124)."""
    return phase * spectrum.spectral_modulation


def phase_change(field: Field, phase, spectrally_modulate: bool = True) -> Field:
    """``u * exp(1j * phase * lambda0/lambda)``.  On a lazily built point
    source the mask is folded into the fused PSF loader."""
    from .sources import LazySourceField

    ny, nx = field.spatial_shape
    if tuple(np.shape(phase))[-2:] != (ny, nx):
        raise AssertionError("Phase must have same height and width as incoming ``Field``.")
    if isinstance(field, LazySourceField) and field.stage == "source":
        return field.with_phase(phase, spectrally_modulate)
    torch = nat.torch_mod()
    from .sources import materialize

    field = materialize(field)
    ph = phase if isinstance(phase, torch.Tensor) else torch.as_tensor(np.asarray(phase, dtype=np.float32))
    ph = ph.to(device=field.device, dtype=torch.float32)
    if field.chromatic:
        mod = torch.as_tensor(field.spectrum.spectral_modulation if spectrally_modulate
                              else np.ones(field.n_wv), dtype=torch.float32, device=field.device)
        ph = ph[..., None] * mod
    return field.replace(u=field.u * torch.polar(torch.ones_like(ph), ph))
