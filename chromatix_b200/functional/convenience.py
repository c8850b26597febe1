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
        ("in_plane", "<i4"), ("conj", "<i4"), ("pupil_out_r2", "<f8"),
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


def _optfft_adjoint_planes(planes: np.ndarray) -> np.ndarray:
    """Plane table of the adjoint optical FFT.

    Per plane the forward map is out = c_out post C(F(pre C(c_in pupil u)))
    (C = conjugation when ``conj``, F the centred DFT).  Its adjoint is the same
    kernel with the grids' roles swapped: input chirp conj(c_out), output chirp
    conj(c_in), the pupil moved to the output grid, ``conj`` flipped, and
    pre' = post, post' = conj(pre) (conj = 0) or pre' = conj(post), post' = pre
    (conj = 1)."""
    a = planes.copy()
    pre = planes["pre_re"] + 1j * planes["pre_im"]
    post = planes["post_re"] + 1j * planes["post_im"]
    c = planes["conj"].astype(bool)
    pre2 = np.where(c, np.conj(post), post)
    post2 = np.where(c, pre, np.conj(pre))
    a["pre_re"], a["pre_im"] = pre2.real, pre2.imag
    a["post_re"], a["post_im"] = post2.real, post2.imag
    a["chirp_in"], a["chirp_out"] = -planes["chirp_out"], -planes["chirp_in"]
    a["dy_in"], a["dx_in"] = planes["dy_out"], planes["dx_out"]
    a["dy_out"], a["dx_out"] = planes["dy_in"], planes["dx_in"]
    a["pupil_out_r2"] = np.where(planes["pupil_r2"] >= 0, np.maximum(planes["pupil_r2"], 1e-300), -1.0)
    a["pupil_r2"] = np.where(planes["pupil_out_r2"] > 0, planes["pupil_out_r2"], -1.0)
    a["conj"] = 1 - planes["conj"]
    a["in_plane"] = np.arange(planes.size)
    return a


class _OptPlan:
    """One ``cx_optical_fft`` call; ``adjoint()`` gives the plan of its gradient."""

    def __init__(self, desc, planes, in_shape, out_shape):
        self.desc, self.planes, self.in_shape, self.out_shape = desc, planes, tuple(in_shape), tuple(out_shape)

    def adjoint(self) -> "_OptPlan":
        d = cx_optfft_desc.from_buffer_copy(self.desc)
        Py, Px = d.ny + 2 * d.pad_y, d.nx + 2 * d.pad_x
        d.ny, d.nx = Py - 2 * d.crop_y, Px - 2 * d.crop_x
        d.pad_y, d.pad_x, d.crop_y, d.crop_x = d.crop_y, d.crop_x, d.pad_y, d.pad_x
        d.n_in_planes = d.n_out_planes
        return _OptPlan(d, _optfft_adjoint_planes(self.planes), self.out_shape, self.in_shape)


def _launch_optfft(plan: _OptPlan, u):
    torch = nat.torch_mod()
    L = _sigs(nat.lib())
    dev = u.device

    def ws_query(d):
        ws_b = nat.c_size_t(0)
        nat.check(L.cx_optfft_workspace_size(d, ws_b))
        return ws_b.value

    ws_bytes, planes_dev = nat.device_table(plan.desc, plan.planes, dev, ws_query)
    u_out = torch.empty(plan.out_shape, dtype=torch.complex64, device=dev)
    ws = nat.workspace(ws_bytes, dev)
    u_in = u.contiguous()
    nat.check(L.cx_optical_fft(plan.desc, nat.ptr(planes_dev), nat.ptr(u_in), nat.ptr(u_out), nat.ptr(ws),
                               ws_bytes, nat.stream_handle(dev)))
    return u_out


_OPT_FN = None


def _opt_fn():
    """torch autograd Function over ``cx_optical_fft``; the backward is the
    adjoint optical FFT (the gradient jax.grad takes through
    functional/convenience.py:9-59 and lenses.py:64-95)."""
    global _OPT_FN
    if _OPT_FN is None:
        torch = nat.torch_mod()

        class _OptFFT(torch.autograd.Function):
            @staticmethod
            def forward(ctx, u, plan):
                ctx.plan = plan
                return _launch_optfft(plan, u)

            @staticmethod
            def backward(ctx, g):
                return _launch_optfft(ctx.plan.adjoint(), g.to(torch.complex64)), None

        _OPT_FN = _OptFFT
    return _OPT_FN


def run_optfft(field: Field, z: float, n: float, pad_width=(0, 0), crop_width=(0, 0), post=1.0 + 0j,
               chirp_in=None, chirp_out=None, pupil_D=None, precision=None):
    """Launch the chirped optical FFT; returns (u_out, du (wv, 2))."""
    nat.require_cuda(field.u, "Field.u")
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
    # one row per wavelength, repeated for every batch element (plane q = b W + w)
    row = np.zeros(W, dtype=FFT_PLANE_DTYPE)
    for w in range(W):
        pre, conj, du, L_sq = norms[w]
        p = row[w]
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
        p["pupil_out_r2"] = -1.0
        p["conj"] = conj
    planes = np.tile(row, nb)
    planes["in_plane"] = np.arange(nb * W)
    d = cx_optfft_desc()
    d.ny, d.nx, d.pad_y, d.pad_x, d.crop_y, d.crop_x = ny, nx, py_, px_, cy, cx
    d.n_wv, d.n_in_planes, d.n_out_planes = W, nb * W, nb * W
    d.precision = config.precision_code(prec)
    oy, ox = Py - 2 * cy, Px - 2 * cx
    out_shape = tuple(B) + (oy, ox) + ((W,) if field.chromatic else ())
    plan = _OptPlan(d, planes, tuple(field.u.shape), out_shape)
    if nat.wants_grad(field.u):
        u_out = _opt_fn().apply(field.u, plan)
    else:
        u_out = _launch_optfft(plan, field.u)
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
