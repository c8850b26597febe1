"""Phase masks (functional/phase_masks.py:29-68, 105-124)."""

from __future__ import annotations

import numpy as np

from .. import _native as nat
from ..core.field import Field

__all__ = ["phase_change", "spectrally_modulate_phase"]


def spectrally_modulate_phase(phase, spectrum):
    """phase * lambda0 / lambda (functional/phase_masks.py:105-124)."""
    return phase * spectrum.spectral_modulation


def channel_scale(field: Field, per_wavelength) -> np.ndarray:
    """A per-wavelength factor repeated over the interleaved channels of ``field``
    (wavelengths x vector components), float32."""
    comps = 3 if field.vectorial else 1
    return np.repeat(np.asarray(per_wavelength, dtype=np.float64).reshape(-1), comps).astype(np.float32)


def real_map(field: Field, m, name: str):
    """A real (ny, nx) map -- or one per batch element -- as a float32 device
    tensor for the elementwise kernels; returns (map, map_batched)."""
    torch = nat.torch_mod()
    ny, nx = field.spatial_shape
    t = m if isinstance(m, torch.Tensor) else torch.as_tensor(np.asarray(m, dtype=np.float32))
    t = t.to(device=field.device, dtype=torch.float32)
    if t.ndim == 2:
        return t.contiguous(), 0
    if t.ndim == field.ndim:
        # (batch..., y, x, 1[, 1]) as broadcast by _broadcast_2d_to_spatial: drop the channel axes
        inner = t.shape[field.ndim + field.spatial_dims[1] + 1:]
        if any(int(v) != 1 for v in inner):
            raise NotImplementedError(f"{name} varying over wavelengths or components is not supported")
        t = t.reshape(t.shape[: field.ndim + field.spatial_dims[1] + 1])
    B = field.batch_shape
    t = t.expand(tuple(B) + (ny, nx)).contiguous()
    return t, 1


_PHASE_FN = None


def _ew_desc(field: Field, batched: int):
    from ..core.field import _channels

    ny, nx = field.spatial_shape
    B = field.batch_shape
    return nat.cx_ew_desc(n_batch=int(np.prod(B)) if B else 1, ny=ny, nx=nx, n_wv=_channels(field),
                          map_batched=batched)


def _phase_fn():
    """autograd Function of ``cx_phase_change``; the backward is
    ``cx_phase_change_adjoint`` (gradients of the field and of the mask)."""
    global _PHASE_FN
    if _PHASE_FN is None:
        torch = nat.torch_mod()

        class _PhaseChange(torch.autograd.Function):
            @staticmethod
            def forward(ctx, u, ph, s, d_bytes):
                d = nat.cx_ew_desc.from_buffer_copy(d_bytes)
                out = torch.empty_like(u)
                nat.check(nat.lib().cx_phase_change(d, nat.ptr(u), nat.ptr(ph), nat.ptr(s), nat.ptr(out),
                                                    nat.stream_handle(u.device)))
                ctx.d_bytes = d_bytes
                ctx.save_for_backward(out, ph, s)
                return out

            @staticmethod
            def backward(ctx, g):
                out, ph, s = ctx.saved_tensors
                d = nat.cx_ew_desc.from_buffer_copy(ctx.d_bytes)
                g = g.to(torch.complex64).contiguous()
                need_u, need_ph = ctx.needs_input_grad[0], ctx.needs_input_grad[1]
                gu = torch.empty_like(g) if need_u else None
                gph = torch.empty_like(ph) if need_ph else None
                nat.check(nat.lib().cx_phase_change_adjoint(d, nat.ptr(g), nat.ptr(out), nat.ptr(ph), nat.ptr(s),
                                                            nat.ptr(gu), nat.ptr(gph), nat.stream_handle(g.device)))
                return gu, gph, None, None

        _PHASE_FN = _PhaseChange
    return _PHASE_FN


def phase_change(field: Field, phase, spectrally_modulate: bool = True) -> Field:
    """``u * exp(1j * phase * lambda0/lambda)`` (functional/phase_masks.py:29-68),
    one pass of the native kernel ``cx_phase_change``.  On a lazily built point
    source the mask is folded into the fused PSF loader."""
    from .sources import LazySourceField

    ny, nx = field.spatial_shape
    if tuple(np.shape(phase))[-2:] != (ny, nx) and not (
            np.ndim(phase) == field.ndim and tuple(np.shape(phase))[field.ndim + field.spatial_dims[0]:][:2] == (ny, nx)):
        raise AssertionError("Phase must have same height and width as incoming ``Field``.")
    torch = nat.torch_mod()
    if isinstance(field, LazySourceField) and field.stage == "source" and not nat.wants_grad(phase):
        return field.with_phase(phase, spectrally_modulate)
    from .sources import materialize

    field = materialize(field)
    nat.require_cuda(field.u, "Field.u")
    ph, batched = real_map(field, phase, "phase")
    mod = field.spectrum.spectral_modulation if (spectrally_modulate and field.chromatic) else np.ones(field.n_wv)
    s = torch.as_tensor(channel_scale(field, mod), device=field.device)
    u = field.u.to(torch.complex64).contiguous()
    d = _ew_desc(field, batched)
    if nat.wants_grad(u, ph):
        out = _phase_fn().apply(u, ph, s, bytes(d))
    else:
        out = torch.empty_like(u)
        nat.check(nat.lib().cx_phase_change(d, nat.ptr(u), nat.ptr(ph), nat.ptr(s), nat.ptr(out),
                                            nat.stream_handle(u.device)))
    return field.replace(u=out)
