"""Rescaled-output propagation: the CZT branch of ``kernel_propagate``
(functional/propagation.py:395-443), reached from ``asm_propagate`` /
``transfer_propagate`` with ``output_dx`` / ``output_shape``.

  Y = fftshift(H * fft2(ifftshift(pad(u))))      one fused optical-FFT call
  Y = CZT_y(Y) * w_y^(-N k) a_y^N                  fused Bluestein pass (column tiles)
  u = CZT_x(Y) * w_x^(-N k) a_x^N / (alpha_y alpha_x)   fused Bluestein pass
with a = exp(-2 pi i lo / T), w = exp(2 pi i (hi - lo) / (T (m - 1))) from the
output grid limits, T the padded input extent and alpha = dx_out / df_in.
"""

from __future__ import annotations

import numpy as np

from .. import _native as nat
from .. import config
from ..core.field import Field, crop, shift_grid
from ..utils.czt import czt_axis
from .convenience import FFT_PLANE_DTYPE, _sigs, cx_optfft_desc


def _spectrum_with_h(field: Field, H, pad: tuple, precision: str):
    """fftshift(H * fft2(ifftshift(pad(u)))) (propagation.py:414-418)."""
    torch = nat.torch_mod()
    L = _sigs(nat.lib())
    if not hasattr(L, "_cx_optical_fft_h_sig"):
        L.cx_optical_fft_h.restype = nat.c_int32
        L.cx_optical_fft_h.argtypes = [nat.ctypes.POINTER(cx_optfft_desc), nat.c_void_p, nat.c_void_p, nat.c_void_p,
                                       nat.c_void_p, nat.c_void_p, nat.c_size_t, nat.c_void_p]
        L._cx_optical_fft_h_sig = True
    ny, nx = field.spatial_shape
    py, px = ny + 2 * pad[0], nx + 2 * pad[1]
    W = field.n_wv
    B = field.batch_shape
    nb = int(np.prod(B)) if B else 1
    planes = np.zeros(nb * W, dtype=FFT_PLANE_DTYPE)
    planes["pre_re"] = 1.0
    planes["post_re"] = 1.0
    planes["pupil_r2"] = -1.0
    planes["dy_in"] = planes["dx_in"] = planes["dy_out"] = planes["dx_out"] = 1.0
    planes["in_plane"] = np.arange(nb * W)
    # H: one plane per output plane, in FFT order (a single plane is shared by the batch)
    Hp = H.reshape(-1, py, px)
    if Hp.shape[0] == 1 and nb * W > 1:
        Hp = Hp.expand(nb * W, py, px)
    Hp = Hp.contiguous()
    d = cx_optfft_desc()
    d.ny, d.nx, d.pad_y, d.pad_x, d.crop_y, d.crop_x = ny, nx, pad[0], pad[1], 0, 0
    d.n_wv, d.n_in_planes, d.n_out_planes = W, nb * W, nb * W
    d.precision = config.precision_code(precision)
    ws_b = nat.c_size_t(0)
    nat.check(L.cx_optfft_workspace_size(d, ws_b))
    out = torch.empty(tuple(B) + (py, px) + ((W,) if field.chromatic else ()), dtype=torch.complex64,
                      device=field.device)
    ws = nat.workspace(ws_b.value, field.device)
    pd = nat.to_device_bytes(planes, field.device)
    nat.check(L.cx_optical_fft_h(d, nat.ptr(pd), nat.ptr(Hp), nat.ptr(field.u.contiguous()), nat.ptr(out),
                                 nat.ptr(ws), ws_b.value, nat.stream_handle(field.device)))
    return out


def rescaled_propagate(field: Field, kernel: int, z, n, pad_width, kykx=(0.0, 0.0), shift_yx=(0.0, 0.0),
                       output_dx=None, output_shape=None, use_czt=True, mode="full", remove_evanescent=False,
                       bandlimit=False, cval=0, precision=None) -> Field:
    from .propagation import _fill_propagator, _pad_tuple

    prec = precision or config.get_precision()
    if cval != 0:
        raise NotImplementedError("non-zero cval padding is not supported by the fused loader")
    if not use_czt:
        raise NotImplementedError("the Yu et al. rescaling branch (use_czt=False) is not part of this build")
    if field.n_wv != 1:
        # the reference indexes the padded extent per axis with T[d] (propagation.py:424-433),
        # which is only meaningful for a single wavelength
        raise NotImplementedError("rescaled (CZT) propagation supports single-wavelength fields")
    if np.asarray(z).size != 1:
        raise NotImplementedError("rescaled (CZT) propagation takes a scalar z")
    z = float(np.asarray(z).reshape(()))
    pad = _pad_tuple(pad_width)
    ny, nx = field.spatial_shape
    py, px = ny + 2 * pad[0], nx + 2 * pad[1]
    if not bandlimit:
        return _rescaled_one_call(field, kernel, z, n, pad, kykx, shift_yx, output_dx, output_shape, mode,
                                  remove_evanescent, pad_width, prec)
    # propagator of the padded field (asm: shift handled by the CZT grid, not in H)
    if kernel == nat.CX_KERNEL_ASM:
        H = _fill_propagator(field, kernel, z, n, kykx, (0.0, 0.0), bandlimit, remove_evanescent, prec, shape=(py, px))
    else:
        H = _fill_propagator(field, kernel, z, n, kykx, precision=prec, shape=(py, px))
    Y = _spectrum_with_h(field, H, pad, prec)
    # output field (propagation.py:396-410)
    m = (py, px) if output_shape is None else (int(output_shape[0]), int(output_shape[1]))
    dx_in = field.dx_wv[0]
    if output_dx is None:
        dx_out = dx_in.copy()
    else:
        if np.ndim(output_dx) != np.ndim(field.dx):
            # Field.empty_like (core/field.py:333-337)
            raise AssertionError("New spacing must have same number of dimensions as old spacing")
        dx_out = np.asarray(output_dx, dtype=np.float64).reshape(-1, 2)[0].copy()
    sh = np.broadcast_to(np.asarray(shift_yx, dtype=np.float64).reshape(-1), (2,))
    T = dx_in * np.array([py, px], dtype=np.float64)  # padded input extent
    alpha = dx_out * T  # dx_out / df_in
    spatial = (-3, -2) if field.chromatic else (-2, -1)
    u = Y
    for d in range(2):
        lo = dx_out[d] * (0 - m[d] / 2) + sh[d]
        hi = dx_out[d] * (m[d] - 1 - m[d] / 2) + sh[d]
        a = np.exp(-1j * 2 * np.pi / T[d] * lo)
        w = np.exp(1j * (2 * np.pi / T[d]) * (hi - lo) / (m[d] - 1))
        N = (m[d] - 1) // 2
        scale = 1.0 / float(np.prod(alpha)) if d == 1 else 1.0
        u = czt_axis(u, m[d], a, w, axis=u.ndim + spatial[d], mod_n=N, scale=scale)
    out = shift_grid(field, sh)
    dx_new = dx_out.reshape(field.dx.shape) if np.size(field.dx) == 2 else np.broadcast_to(dx_out, field.dx.shape)
    out = out.replace(u=u, dx=np.array(dx_new, dtype=np.float64))
    if mode == "same":
        out = crop(out, pad_width)
    return out


class cx_czt_prop_desc(nat.ctypes.Structure):
    _fields_ = [(k, nat.c_int32) for k in ("ny", "nx", "pad_y", "pad_x", "my", "mx", "n_fields", "kernel",
                                           "precision", "remove_evanescent", "bandlimit", "reserved")] + \
               [(k, nat.c_double) for k in ("n_medium", "z", "wavelength", "dy_in", "dx_in", "dy_out", "dx_out",
                                            "shift_y", "shift_x", "ky0", "kx0")]


def _czt_prop_sigs(L):
    if not hasattr(L, "_cx_czt_propagate_sig"):
        P = nat.ctypes.POINTER(cx_czt_prop_desc)
        L.cx_czt_propagate_workspace_size.restype = nat.c_int32
        L.cx_czt_propagate_workspace_size.argtypes = [P, nat.ctypes.POINTER(nat.c_size_t)]
        L.cx_czt_propagate.restype = nat.c_int32
        L.cx_czt_propagate.argtypes = [P, nat.c_void_p, nat.c_void_p, nat.c_void_p, nat.c_size_t, nat.c_void_p]
        L._cx_czt_propagate_sig = True
    return L


def _rescaled_one_call(field: Field, kernel, z, n, pad, kykx, shift_yx, output_dx, output_shape, mode,
                       remove_evanescent, pad_width, prec) -> Field:
    """The whole CZT branch as one native call (``cx_czt_propagate``)."""
    torch = nat.torch_mod()
    L = _czt_prop_sigs(nat.lib())
    ny, nx = field.spatial_shape
    py, px = ny + 2 * pad[0], nx + 2 * pad[1]
    m = (py, px) if output_shape is None else (int(output_shape[0]), int(output_shape[1]))
    dx_in = field.dx_wv[0]
    if output_dx is None:
        dx_out = dx_in.copy()
    else:
        if np.ndim(output_dx) != np.ndim(field.dx):
            # Field.empty_like (core/field.py:333-337)
            raise AssertionError("New spacing must have same number of dimensions as old spacing")
        dx_out = np.asarray(output_dx, dtype=np.float64).reshape(-1, 2)[0].copy()
    sh = np.broadcast_to(np.asarray(shift_yx, dtype=np.float64).reshape(-1), (2,))
    B = field.batch_shape
    nb = int(np.prod(B)) if B else 1
    d = cx_czt_prop_desc()
    d.ny, d.nx, d.pad_y, d.pad_x = ny, nx, pad[0], pad[1]
    d.my, d.mx = m
    d.n_fields = nb
    d.kernel = kernel
    d.precision = config.precision_code(prec)
    d.remove_evanescent = int(bool(remove_evanescent))
    d.n_medium, d.z, d.wavelength = float(n), float(z), float(field.spectrum.wavelength[0])
    d.dy_in, d.dx_in = float(dx_in[0]), float(dx_in[1])
    d.dy_out, d.dx_out = float(dx_out[0]), float(dx_out[1])
    d.shift_y, d.shift_x = float(sh[0]), float(sh[1])
    ky0, kx0 = np.asarray(kykx, dtype=np.float64).reshape(2)
    d.ky0, d.kx0 = float(ky0), float(kx0)
    wsb = nat.c_size_t(0)
    nat.check(L.cx_czt_propagate_workspace_size(d, wsb))
    ws = nat.workspace(wsb.value, field.device)
    u_in = field.u.contiguous()
    spatial_last = not field.chromatic
    u = torch.empty(tuple(B) + tuple(m) + (() if spatial_last else (1,)), dtype=torch.complex64,
                    device=field.device)
    nat.check(L.cx_czt_propagate(d, nat.ptr(u_in), nat.ptr(u), nat.ptr(ws), wsb.value,
                                 nat.stream_handle(field.device)))
    out = shift_grid(field, sh)
    dx_new = dx_out.reshape(field.dx.shape) if np.size(field.dx) == 2 else np.broadcast_to(dx_out, field.dx.shape)
    out = out.replace(u=u, dx=np.array(dx_new, dtype=np.float64))
    if mode == "same":
        out = crop(out, pad_width)
    return out
