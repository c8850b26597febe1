"""Rescaled-output propagation: the CZT branch of ``kernel_propagate``
(functional/propagation.py:395-443), reached from ``asm_propagate`` /
``transfer_propagate`` with ``output_dx`` / ``output_shape``.

  Y = fftshift(H * fft2(ifftshift(pad(u))))      optical-FFT pass with the propagator table
  Y = CZT_y(Y) * w_y^(-N k) a_y^N                  fused Bluestein pass (column tiles)
  u = CZT_x(Y) * w_x^(-N k) a_x^N / (alpha_y alpha_x)   fused Bluestein pass
all in one native call (``cx_czt_propagate``),
with a = exp(-2 pi i lo / T), w = exp(2 pi i (hi - lo) / (T (m - 1))) from the
output grid limits, T the padded input extent and alpha = dx_out / df_in.
With ``use_czt=False`` the two chirp-Z passes are replaced by the Yu et al.
chirp convolution (propagation.py:445-458), run by the same fused passes in
their convolution mode; its output keeps the padded grid's shape.
"""

from __future__ import annotations

import numpy as np

from .. import _native as nat
from .. import config
from ..core.field import Field, crop, shift_grid


def rescaled_propagate(field: Field, kernel: int, z, n, pad_width, kykx=(0.0, 0.0), shift_yx=(0.0, 0.0),
                       output_dx=None, output_shape=None, use_czt=True, mode="full", remove_evanescent=False,
                       bandlimit=False, cval=0, precision=None) -> Field:
    from .propagation import _pad_tuple

    prec = precision or config.get_precision()
    nat.refuse_grad("rescaled (output_dx / output_shape) propagation", field.u)
    if field.n_wv != 1:
        # the reference indexes the padded extent per axis with T[d] (propagation.py:424-433),
        # which is only meaningful for a single wavelength
        raise NotImplementedError("rescaled (CZT) propagation supports single-wavelength fields")
    if np.asarray(z).size != 1:
        raise NotImplementedError("rescaled (CZT) propagation takes a scalar z")
    z = float(np.asarray(z).reshape(()))
    pad = _pad_tuple(pad_width)
    if cval != 0 and (pad[0] or pad[1]):
        # constant padding by the native pad kernel; the padded grid is the same
        from ..core.field import pad as pad_field

        field = pad_field(field, pad, cval)
        pad = (0, 0)
    return _rescaled_one_call(field, kernel, z, n, pad, kykx, shift_yx, output_dx, output_shape, mode,
                              remove_evanescent, pad_width, prec, method=0 if use_czt else 1,
                              bandlimit=bool(bandlimit) and kernel == nat.CX_KERNEL_ASM)


class cx_czt_prop_desc(nat.ctypes.Structure):
    _fields_ = [(k, nat.c_int32) for k in ("ny", "nx", "pad_y", "pad_x", "my", "mx", "n_fields", "kernel",
                                           "precision", "remove_evanescent", "bandlimit", "method")] + \
               [(k, nat.c_double) for k in ("n_medium", "z", "wavelength", "dy_in", "dx_in", "dy_out", "dx_out",
                                            "shift_y", "shift_x", "ky0", "kx0", "bl_y0", "bl_x0", "bl_hy", "bl_hx")]


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
                       remove_evanescent, pad_width, prec, method: int = 0, bandlimit: bool = False) -> Field:
    """The whole rescaled branch as one native call (``cx_czt_propagate``):
    method 0 = chirp-Z transforms, 1 = the Yu et al. chirp convolution."""
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
    d.method = int(method)
    d.n_medium, d.z, d.wavelength = float(n), float(z), float(field.spectrum.wavelength[0])
    d.dy_in, d.dx_in = float(dx_in[0]), float(dx_in[1])
    d.dy_out, d.dx_out = float(dx_out[0]), float(dx_out[1])
    d.shift_y, d.shift_x = float(sh[0]), float(sh[1])
    ky0, kx0 = np.asarray(kykx, dtype=np.float64).reshape(2)
    d.ky0, d.kx0 = float(ky0), float(kx0)
    if bandlimit:
        from .propagation import _bandlimit_rect

        # asm_propagate passes shift_yx to the propagator only without chirp-Z (propagation.py:331-339)
        bsh = (float(sh[0]), float(sh[1])) if method == 1 else (0.0, 0.0)
        k0, km = _bandlimit_rect(float(z), float(field.spectrum.wavelength[0]), bsh, float(dx_in[0]),
                                 float(dx_in[1]), py, px, prec)
        d.bandlimit = 1
        d.bl_y0, d.bl_x0 = (float(v) for v in k0)
        d.bl_hy, d.bl_hx = (float(v) for v in km)
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
