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


def _apply(field: Field, kind: int, params) -> Field:
    """One pass of the native pupil kernel ``cx_pupil``; ``params`` per
    wavelength: (p0, p1, p2, p3) as documented in include/cx_b200.h."""
    from .phase_masks import _ew_desc
    from .sources import materialize

    torch = nat.torch_mod()
    field = materialize(field)
    nat.require_cuda(field.u, "Field.u")
    W = field.n_wv
    comps = 3 if field.vectorial else 1
    dxw = field.dx_wv
    rows = []
    for w in range(W):
        p = [float(v) for v in np.broadcast_to(np.asarray(params[min(w, len(params) - 1)], np.float64), (4,))]
        rows += [[dxw[w, 0], dxw[w, 1]] + p] * comps
    tab = nat.upload(np.asarray(rows, dtype=np.float64), field.device)
    org = np.asarray(field.origin, dtype=np.float64).reshape(-1, 2)[0]
    u = field.u.to(torch.complex64).contiguous()
    args = (bytes(_ew_desc(field, 0)), int(kind), tab, float(org[0]), float(org[1]))
    if nat.wants_grad(u):
        return field.replace(u=_pupil_fn().apply(u, args))
    return field.replace(u=_pupil_launch(u, *args))


def _pupil_launch(u, d_bytes, kind, tab, oy, ox):
    torch = nat.torch_mod()
    out = torch.empty_like(u)
    nat.check(nat.lib().cx_pupil(nat.cx_ew_desc.from_buffer_copy(d_bytes), kind, nat.ptr(tab), oy, ox, nat.ptr(u),
                                 nat.ptr(out), nat.stream_handle(u.device)))
    return out


_PUPIL_FN = None


def _pupil_fn():
    """autograd Function of the native pupil: a real mask is its own adjoint."""
    global _PUPIL_FN
    if _PUPIL_FN is None:
        torch = nat.torch_mod()

        class _Pupil(torch.autograd.Function):
            @staticmethod
            def forward(ctx, u, args):
                ctx.args = args
                return _pupil_launch(u, *args)

            @staticmethod
            def backward(ctx, g):
                return _pupil_launch(g.to(torch.complex64).contiguous(), *ctx.args), None

        _PUPIL_FN = _Pupil
    return _PUPIL_FN


def _scale(field: Field):
    return field.spectrum.central_wavelength / np.asarray(field.spectrum.wavelength, dtype=np.float64)


def circular_pupil(field: Field, w) -> Field:
    """|r|^2 <= ((lam0/lam) w / 2)^2 (functional/pupils.py:17-23)."""
    return _apply(field, 0, [(r, 0, 0, 0) for r in _scale(field) * w / 2])


def square_pupil(field: Field, w) -> Field:
    """max(|y|, |x|) <= (lam0/lam) w / 2 (functional/pupils.py:26-31)."""
    return _apply(field, 1, [(r, 0, 0, 0) for r in _scale(field) * w / 2])


def super_gaussian_pupil(field: Field, w, n=16) -> Field:
    """exp(-(|r| / w)^n) (functional/pupils.py:49-55)."""
    return _apply(field, 2, [(float(w), float(n), 0, 0)])


def tukey_pupil(field: Field, w) -> Field:
    """Tukey window (functional/pupils.py:58-67): alpha = w / max|extent| per
    wavelength on r = |g / extent| clipped to [0, 1/2]."""
    ext = np.asarray(field.extent, dtype=np.float64).reshape(-1, 2)
    alpha = w / np.max(np.abs(ext), axis=-1)
    return _apply(field, 3, [(0.0, float(alpha[k]), float(ext[k, 0]), float(ext[k, 1])) for k in range(ext.shape[0])])
