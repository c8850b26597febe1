"""Centred optical FFT (functional/convenience.py:9-59) and its chirped variants.

All of them run through ``cx_optical_fft``: padding, input chirp, pupil,
normalisation and the z < 0 conjugation are evaluated in the FFT loader,
fftshift/ifftshift are index remaps, and the output chirp and crop happen in
the store.
"""

from __future__ import annotations

import numpy as np

from .. import _native as nat
from .. import config
from ..core.field import Field

FFT_PLANE_DTYPE = np.dtype(
    [
        ("pre_re", "<f8"), ("pre_im", "<f8"), ("post_re", "<f8"), ("post_im", "<f8"),
        ("chirp_in", "<f8"), ("chirp_out", "<f8"), ("dy_in", "<f8"), ("dx_in", "<f8"),
        ("dy_out", "<f8"), ("dx_out", "<f8"), ("oy", "<f8"), ("ox", "<f8"), ("pupil_r2", "<f8"),
        ("in_plane", "<i4"), ("conj", "<i4"),
    ]
)


class cx_optfft_desc(nat.ctypes.Structure):
    _fields_ = [(n, nat.c_int32) for n in
                ("ny", "nx", "pad_y", "pad_x", "crop_y", "crop_x", "n_wv", "n_in_planes", "n_out_planes",
                 "precision")]


_SIGS_DONE = False


def _sigs(L):
    global _SIGS_DONE
    if not _SIGS_DONE:
        L.cx_optfft_workspace_size.restype = nat.c_int32
        L.cx_optfft_workspace_size.argtypes = [nat.ctypes.POINTER(cx_optfft_desc), nat.ctypes.POINTER(nat.c_size_t)]
        L.cx_optical_fft.restype = nat.c_int32
        L.cx_optical_fft.argtypes = [nat.ctypes.POINTER(cx_optfft_desc), nat.c_void_p, nat.c_void_p, nat.c_void_p,
                                     nat.c_void_p, nat.c_size_t, nat.c_void_p]
        _SIGS_DONE = True
    return L


def _optfft_norms(field: Field, z: float, n: float, shape):
    """Per-wavelength (pre factor, conj flag, du) of optical_fft (convenience.py:33-58)."""
    ny, nx = shape
    dxw = field.dx_wv
    out = []
    for w in range(field.n_wv):
        lam = field.spectrum.wavelength[w]
        L_sq = lam * z / n
        du = np.array([1.0 / (ny * dxw[w, 0]), 1.0 / (nx * dxw[w, 1])]) * abs(L_sq)
        if z >= 0:
            pre = -1j * dxw[w, 0] * dxw[w, 1] / L_sq
            conj = 0
        else:
            pre = -1j * (L_sq / (du[0] * du[1])) / (ny * nx)
            conj = 1
        out.append((pre, conj, du, L_sq))
    return out


def run_optfft(field: Field, z: float, n: float, pad_width=(0, 0), crop_width=(0, 0), post=1.0 + 0j,
               chirp_in=None, chirp_out=None, pupil_D=None, precision=None):
    """Launch the chirped optical FFT; returns (u_out, du (wv, 2))."""
    torch = nat.torch_mod()
    nat.require_cuda(field.u, "Field.u")
    L = _sigs(nat.lib())
    prec = precision or config.get_precision()
    py_, px_ = pad_width
    cy, cx = crop_width
    ny, nx = field.spatial_shape
    Py, Px = ny + 2 * py_, nx + 2 * px_
    W = field.n_wv
    B = field.batch_shape
    nb = int(np.prod(B)) if B else 1
    norms = _optfft_norms(field, z, n, (Py, Px))
    dxw = field.dx_wv
    org = np.asarray(field.origin, dtype=np.float64).reshape(-1, 2)
    planes = np.zeros(nb * W, dtype=FFT_PLANE_DTYPE)
    for b in range(nb):
        for w in range(W):
            q = b * W + w
            pre, conj, du, L_sq = norms[w]
            p = planes[q]
            p["pre_re"], p["pre_im"] = pre.real, pre.imag
            post_w = complex(post[w] if np.ndim(post) else post)
            p["post_re"], p["post_im"] = post_w.real, post_w.imag
            p["chirp_in"] = 0.0 if chirp_in is None else float(np.atleast_1d(chirp_in)[min(w, np.size(chirp_in) - 1)])
            p["chirp_out"] = 0.0 if chirp_out is None else float(
                np.atleast_1d(chirp_out)[min(w, np.size(chirp_out) - 1)])
            p["dy_in"], p["dx_in"] = dxw[w]
            p["dy_out"], p["dx_out"] = du
            p["oy"], p["ox"] = org[min(w, org.shape[0] - 1)]
            if pupil_D is not None:
                r = (field.spectrum.central_wavelength / field.spectrum.wavelength[w]) * pupil_D / 2
                p["pupil_r2"] = r * r
            else:
                p["pupil_r2"] = -1.0
            p["in_plane"] = q
            p["conj"] = conj
    d = cx_optfft_desc()
    d.ny, d.nx, d.pad_y, d.pad_x, d.crop_y, d.crop_x = ny, nx, py_, px_, cy, cx
    d.n_wv, d.n_in_planes, d.n_out_planes = W, nb * W, nb * W
    d.precision = config.precision_code(prec)
    ws_b = nat.c_size_t(0)
    nat.check(L.cx_optfft_workspace_size(d, ws_b))
    oy, ox = Py - 2 * cy, Px - 2 * cx
    out_shape = tuple(B) + (oy, ox) + ((W,) if field.chromatic else ())
    u_out = torch.empty(out_shape, dtype=torch.complex64, device=field.device)
    ws = nat.workspace(ws_b.value, field.device)
    planes_dev = nat.to_device_bytes(planes, field.device)
    u_in = field.u.contiguous()
    nat.check(L.cx_optical_fft(d, nat.ptr(planes_dev), nat.ptr(u_in), nat.ptr(u_out), nat.ptr(ws), ws_b.value,
                               nat.stream_handle(field.device)))
    du = np.stack([nm[2] for nm in norms])
    return u_out, du


def _dx_like(field: Field, du_wv: np.ndarray):
    return du_wv.reshape(2) if not field.chromatic else du_wv


def optical_fft(field: Field, z, n, *, precision=None) -> Field:
    """``fftshift(fft2(ifftshift(norm * u)))`` with the output spacing
    ``du = df * |lambda z / n|`` (functional/convenience.py:9-59)."""
    from .sources import materialize

    field = materialize(field)
    u, du = run_optfft(field, float(z), float(n), precision=precision)
    return field.replace(u=u, dx=_dx_like(field, du))


def _optical_fft_chirped(field: Field, z, n, pad_width, cval=0, skip_initial_phase=False, skip_final_phase=False,
                         precision=None) -> Field:
    """transform_propagate (functional/propagation.py:34-82) as one fused call."""
    from .sources import materialize

    if cval != 0:
        raise NotImplementedError("non-zero cval padding is not supported by the fused loader")
    field = materialize(field)
    if isinstance(pad_width, (int, np.integer)):
        pad_width = (int(pad_width), int(pad_width))
    z = float(z)
    n = float(n)
    L_sq = field.spectrum.wavelength * z / n
    c = np.pi / L_sq
    u, du = run_optfft(field, z, n, pad_width=tuple(pad_width), crop_width=tuple(pad_width), post=1j,
                       chirp_in=None if skip_initial_phase else c, chirp_out=None if skip_final_phase else c,
                       precision=precision)
    return field.replace(u=u, dx=_dx_like(field, du))
