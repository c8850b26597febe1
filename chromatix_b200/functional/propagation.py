"""Free-space propagation with the same signatures as ``chromatix.functional``.

Reference: functional/propagation.py.  The Fourier-multiplier propagators
(transfer, angular spectrum / exact, explicit kernel) run as one fused
three-pass CUDA pipeline (``cx_prop2d``): zero padding in the first FFT's
loader, the transfer function evaluated on the fly between the column FFT and
IFFT, the crop in the last FFT's store.
"""

from __future__ import annotations

import collections
from typing import Literal

import numpy as np

from .. import _native as nat
from .. import config
from ..core.field import Field, crop, shift_grid

__all__ = [
    "transform_propagate",
    "transform_propagate_sas",
    "transfer_propagate",
    "asm_propagate",
    "kernel_propagate",
    "compute_transfer_propagator",
    "compute_asm_propagator",
    "compute_padding_transform",
    "compute_padding_transfer",
    "compute_padding_exact",
]

_BOUNDARIES = ("tukey", "super_gaussian")


def _pad_tuple(pad_width):
    if isinstance(pad_width, (int, np.integer)):
        return int(pad_width), int(pad_width)
    py, px = pad_width
    return int(py), int(px)


def _z_array(z):
    z = np.asarray(z, dtype=np.float64)
    if z.size > 1:
        return z.reshape(-1), (z.size,)
    return z.reshape(-1)[:1], ()


def _bandlimit_rect(z, lam, shift_yx, dy, dx, py, px, prec: str):
    """Matsushima band-limit rectangle (functional/propagation.py:557-579)."""
    dt = np.float32 if prec == "ref32" else np.float64
    s = np.asarray(shift_yx, dtype=dt)
    ext = np.array([dy * py, dx * px], dtype=dt)
    df = dt(1) / ext
    z = dt(z)
    lam = dt(lam)
    with np.errstate(divide="ignore"):
        klp = ((s + 1 / (2 * df)) ** (-2) * z**2 + 1) ** (-0.5) / lam
        kln = ((s - 1 / (2 * df)) ** (-2) * z**2 + 1) ** (-0.5) / lam
    k0 = 0.5 * (np.sign(s + ext) * klp + np.sign(s - ext) * kln)
    kw = np.sign(s + ext) * klp - np.sign(s - ext) * kln
    return k0.astype(np.float64), (kw / 2).astype(np.float64)


def _plan_planes(field: Field, zs, zshape, py, px, shift_yx=(0.0, 0.0), bandlimit=False, prec="accurate",
                 h_index=None, batch_shape=None):
    """Per-output-plane launch parameters.

    Output batch = broadcast(field batch, z batch) as in the reference
    (z broadcast to the innermost batch, utils/shapes.py:52-58).
    """
    B = field.batch_shape if batch_shape is None else tuple(batch_shape)
    out_batch = np.broadcast_shapes(B, zshape)
    nb_in = int(np.prod(B)) if B else 1
    nb_out = int(np.prod(out_batch)) if out_batch else 1
    in_idx = np.broadcast_to(np.arange(nb_in).reshape(B if B else ()), out_batch).reshape(-1)
    if zshape:
        z_idx = np.broadcast_to(np.arange(zs.size).reshape(zshape), out_batch).reshape(-1)
    else:
        z_idx = np.zeros(nb_out, dtype=np.int64)
    W = field.n_wv
    dxw = np.asarray(field.dx_wv, dtype=np.float64).reshape(W, 2)
    wl = np.asarray(field.spectrum.wavelength, dtype=np.float64).reshape(W)
    planes = np.zeros(nb_out * W, dtype=nat.PLANE_DTYPE)
    sy, sx = np.asarray(shift_yx, dtype=np.float64).reshape(2)
    # plane q = ob W + w (batch-major, channel innermost)
    zq = np.repeat(np.asarray(zs, dtype=np.float64).reshape(-1)[z_idx], W)
    planes["z"] = zq
    planes["wavelength"] = np.tile(wl, nb_out)
    planes["dy"] = np.tile(dxw[:, 0], nb_out)
    planes["dx"] = np.tile(dxw[:, 1], nb_out)
    planes["shift_y"] = sy
    planes["shift_x"] = sx
    planes["in_plane"] = (np.repeat(in_idx.astype(np.int64), W) * W + np.tile(np.arange(W), nb_out))
    if h_index is not None:
        planes["h_plane"] = np.asarray(h_index, dtype=np.int64).reshape(-1)[: nb_out * W]
    if bandlimit:
        for q in range(nb_out * W):
            w = q % W
            k0, km = _bandlimit_rect(float(zq[q]), wl[w], (sy, sx), dxw[w, 0], dxw[w, 1], py, px, prec)
            planes[q]["bl_y0"], planes[q]["bl_x0"] = k0
            planes[q]["bl_hy"], planes[q]["bl_hx"] = km
    return planes, out_batch, nb_in, nb_out


class _PropPlan:
    """One ``cx_prop2d`` call: descriptor, plane table, input and output shapes.

    ``adjoint()`` returns the plan of the gradient: the same fused passes with
    conj(H) (= H(-z) for the transfer and ASM kernels), reading the output
    gradient plane by plane; zero padding becomes a crop.  Output planes that
    share an input (z broadcast over the field batch) are summed afterwards."""

    def __init__(self, desc, planes, in_shape, out_shape, chromatic: bool, H=None):
        self.desc, self.planes, self.H = desc, planes, H
        self.in_shape, self.out_shape, self.chromatic = tuple(in_shape), tuple(out_shape), bool(chromatic)

    def adjoint(self) -> "_PropPlan":
        d = nat.cx_prop2d_desc.from_buffer_copy(self.desc)
        py, px = d.ny + 2 * d.pad_y, d.nx + 2 * d.pad_x
        ny, nx = d.ny, d.nx
        if not d.mode_same:
            d.ny, d.nx = py - 2 * d.crop_y, px - 2 * d.crop_x
            d.pad_y, d.pad_x, d.crop_y, d.crop_x = d.crop_y, d.crop_x, d.pad_y, d.pad_x
        d.n_in_planes = d.n_out_planes
        d.conj_kernel = 1 - d.conj_kernel
        planes = self.planes.copy()
        planes["in_plane"] = np.arange(planes.size)
        spatial = 3 if self.chromatic else 2
        out_batch = self.out_shape[: len(self.out_shape) - spatial]
        adj_out = out_batch + (ny, nx) + ((d.n_wv,) if self.chromatic else ())
        return _PropPlan(d, planes, self.out_shape, adj_out, self.chromatic, self.H)


# propagation call parameters -> (descriptor, plane table, output shape);
# descriptors and tables are never modified after they are built
_HOST_PLANS = collections.OrderedDict()
_PLAN_CACHE_SIZE = 64


def _prop_ws(d) -> int:
    ws = nat.c_size_t(0)
    nat.check(nat.lib().cx_prop2d_workspace_size(d, ws))
    return ws.value


def _launch_prop2d(plan: _PropPlan, u_in):
    torch = nat.torch_mod()
    L = nat.lib()
    d = plan.desc
    dev = u_in.device
    ws_bytes, planes_dev = nat.device_table(d, plan.planes, dev, _prop_ws)
    u_in = u_in.contiguous()
    u_out = torch.empty(plan.out_shape, dtype=torch.complex64, device=dev)
    ws = nat.workspace(ws_bytes, dev)
    nat.check(L.cx_prop2d(d, nat.ptr(planes_dev), nat.ptr(u_in), nat.ptr(u_out), nat.ptr(plan.H), nat.ptr(ws),
                          ws_bytes, nat.stream_handle(dev)))
    return u_out


_PROP_FN = None


def _prop_fn():
    """torch autograd Function over ``cx_prop2d``: forward the fused
    propagation, backward the same kernels with the conjugate propagator (the
    hand-written adjoint of functional/propagation.py:391-394, which the
    reference obtains from jax.grad)."""
    global _PROP_FN
    if _PROP_FN is None:
        torch = nat.torch_mod()

        class _Prop2D(torch.autograd.Function):
            @staticmethod
            def forward(ctx, u, plan):
                ctx.plan = plan
                return _launch_prop2d(plan, u)

            @staticmethod
            def backward(ctx, g):
                plan = ctx.plan
                adj = plan.adjoint()
                gu = _launch_prop2d(adj, g.to(torch.complex64))
                return gu.sum_to_size(plan.in_shape), None

        _PROP_FN = _Prop2D
    return _PROP_FN


def _apply_prop(plan: _PropPlan, u):
    if plan.H is not None:
        nat.refuse_grad("kernel_propagate (gradient with respect to the propagator)", plan.H)
    if nat.wants_grad(u):
        return _prop_fn().apply(u, plan)
    return _launch_prop2d(plan, u)


def _fused_size(n: int) -> bool:
    """Transform lengths of the fused propagation passes (2^a {1, 3, 5, 7} up to 4096, and 8192)."""
    return n == 8192 or bool(nat.lib().cx_fft_size_supported(int(n)))


_CMUL_FN = None


def _cmul_planar(u, H, chromatic: bool):
    """u (B, py, px[, W]) x planar H (B W, py, px) by the native multiplier; its
    gradient with respect to u is g conj(H)."""
    global _CMUL_FN
    torch = nat.torch_mod()

    def launch(x, conj):
        W = x.shape[-1] if chromatic else 1
        py, px = (x.shape[-3], x.shape[-2]) if chromatic else (x.shape[-2], x.shape[-1])
        B = x.numel() // (py * px * W)
        d = nat.cx_ew_desc(n_batch=B, ny=py, nx=px, n_wv=W, map_batched=1)
        out = torch.empty_like(x)
        nat.check(nat.lib().cx_cmul_planar(d, nat.ptr(x), nat.ptr(H), int(conj), nat.ptr(out),
                                           nat.stream_handle(x.device)))
        return out

    if _CMUL_FN is None:
        class _CMul(torch.autograd.Function):
            @staticmethod
            def forward(ctx, x, fn):
                ctx.fn = fn
                return fn(x.contiguous(), False)

            @staticmethod
            def backward(ctx, g):
                return ctx.fn(g.to(torch.complex64).contiguous(), True), None

        _CMUL_FN = _CMul
    if nat.wants_grad(u):
        return _CMUL_FN.apply(u, launch)
    return launch(u.contiguous(), False)


def _prop2d_general(field: Field, kernel: int, zs, zshape, n, pad, kykx, shift_yx, remove_evanescent,
                    bandlimit, mode, crop_w, prec, H=None, h_index=None):
    """kernel_propagate's FFT branch (functional/propagation.py:391-394) on a
    padded grid whose lengths the fused passes do not cover: the 2D DFT and its
    inverse as chirp-Z passes along y and x (an exact length-N DFT by
    Bluestein's algorithm: a = 1, w = exp(-+2 pi i / N)), the propagator from
    ``cx_fill_propagator`` (or the caller's table), the product by the native
    planar multiplier.  Every step is a native kernel with an adjoint."""
    from ..core.field import pad as pad_field
    from ..utils.czt import czt_axis

    torch = nat.torch_mod()
    py_, px_ = pad
    f = pad_field(field, (py_, px_)) if (py_ or px_) else field
    py, px = f.spatial_shape
    W = f.n_wv
    chrom = bool(f.chromatic)
    B = f.batch_shape
    out_batch = tuple(np.broadcast_shapes(B, zshape))
    spatial = (py, px) + ((W,) if chrom else ())
    u = f.u.to(torch.complex64)
    if tuple(B) != out_batch:
        u = u.expand(out_batch + spatial)
    u = u.reshape((-1,) + spatial)
    ay, ax = (-3, -2) if chrom else (-2, -1)
    if H is None:
        Hp = _fill_propagator(f, kernel, zs if zshape else zs[:1], n, kykx, shift_yx, bandlimit, remove_evanescent,
                              precision=prec)
        # (z batch..., [wv,] py, px) -> planar per (output batch element, wavelength)
        Hp = Hp.movedim(-1, -3) if chrom else Hp.unsqueeze(-3)
        Hp = Hp.expand(out_batch + (W, py, px)).reshape(-1, py, px).contiguous()
    else:
        Hp = H[torch.as_tensor(np.asarray(h_index), device=H.device)].contiguous()
    U = czt_axis(czt_axis(u, py, 1.0, np.exp(-2j * np.pi / py), axis=ay), px, 1.0, np.exp(-2j * np.pi / px), axis=ax)
    U = _cmul_planar(U, Hp, chrom)
    out = czt_axis(czt_axis(U, py, 1.0, np.exp(2j * np.pi / py), axis=ay, scale=1.0 / py), px, 1.0,
                   np.exp(2j * np.pi / px), axis=ax, scale=1.0 / px)
    out = out.reshape(out_batch + spatial)
    cy, cx = crop_w
    if cy or cx:
        sl = [slice(None)] * out.ndim
        sl[out.ndim + ay] = slice(cy, py - cy)
        sl[out.ndim + ax] = slice(cx, px - cx)
        out = out[tuple(sl)].contiguous()
    return out


def _pad_const(field: Field, pad_width, cval):
    """Field padded with the constant ``cval`` by the native pad kernel
    (core/field.py:534-549); its gradient is the crop of the output gradient."""
    from ..core.field import pad

    return pad(field, pad_width, cval)


def _run_prop2d(field: Field, kernel: int, zs, zshape, n, pad_width, kykx=(0.0, 0.0), shift_yx=(0.0, 0.0),
                remove_evanescent=False, bandlimit=False, mode="full", H=None, h_index=None, precision=None,
                cval=0.0):
    nat.require_cuda(field.u, "Field.u")
    prec = precision or config.get_precision()
    py_, px_ = _pad_tuple(pad_width)
    crop = (0, 0)
    if cval != 0 and (py_ or px_):
        # explicit constant padding, then the padded field propagates without
        # loader padding; "same" crops the padding off again
        field = _pad_const(field, (py_, px_), cval)
        if mode == "same":
            crop = (py_, px_)
            mode = "full"
        py_, px_ = 0, 0
    ny, nx = field.spatial_shape
    py, px = ny + 2 * py_, nx + 2 * px_
    if not (_fused_size(py) and _fused_size(px)):
        crop_w = (py_, px_) if mode == "same" else crop
        return _prop2d_general(field, kernel, zs, zshape, n, (py_, px_), kykx, shift_yx, remove_evanescent, bandlimit,
                               mode, crop_w, prec, H=H, h_index=h_index)
    W = field.n_wv
    key = (kernel, tuple(field.u.shape), field.batch_shape, W, field.chromatic, py_, px_, crop, mode, prec,
           np.asarray(field.dx_wv, dtype=np.float64).tobytes(),
           np.asarray(field.spectrum.wavelength, dtype=np.float64).tobytes(),
           np.asarray(zs, dtype=np.float64).tobytes(), tuple(zshape), float(n), tuple(np.ravel(kykx).tolist()),
           tuple(np.ravel(shift_yx).tolist()), bool(remove_evanescent), bool(bandlimit),
           None if h_index is None else np.asarray(h_index).tobytes())
    hit = _HOST_PLANS.get(key)
    if hit is not None:
        _HOST_PLANS.move_to_end(key)
        d, planes, out_shape = hit
        return _apply_prop(_PropPlan(d, planes, tuple(field.u.shape), out_shape, field.chromatic, H), field.u)
    planes, out_batch, nb_in, nb_out = _plan_planes(field, zs, zshape, py, px, shift_yx, bandlimit, prec, h_index)
    d = nat.cx_prop2d_desc()
    d.ny, d.nx, d.pad_y, d.pad_x = ny, nx, py_, px_
    d.n_wv = W
    d.n_in_planes = nb_in * W
    d.n_out_planes = nb_out * W
    d.mode_same = 1 if mode == "same" else 0
    d.crop_y, d.crop_x = crop
    d.kernel = kernel
    d.precision = config.precision_code(prec, tensor_core=config.tensor_core_grid(py, px))
    d.remove_evanescent = int(bool(remove_evanescent))
    d.bandlimit = int(bool(bandlimit))
    d.n_medium = float(n)
    ky0, kx0 = np.asarray(kykx, dtype=np.float64).reshape(2)
    d.ky0, d.kx0 = float(ky0), float(kx0)
    oy, ox = (ny, nx) if mode == "same" else (py - 2 * crop[0], px - 2 * crop[1])
    out_shape = tuple(out_batch) + (oy, ox) + ((W,) if field.chromatic else ())
    _HOST_PLANS[key] = (d, planes, out_shape)
    if len(_HOST_PLANS) > _PLAN_CACHE_SIZE:
        _HOST_PLANS.popitem(last=False)
    plan = _PropPlan(d, planes, tuple(field.u.shape), out_shape, field.chromatic, H)
    return _apply_prop(plan, field.u)


def _check_mode(mode):
    if mode not in ("full", "same"):
        raise ValueError(f"mode must be 'full' or 'same', got {mode!r}")


def _check_boundary(absorbing_boundary):
    # kernel_propagate applies the pupil to the pre-propagation field object and
    # then returns field.replace(u=u): the boundary never reaches the output
    # (functional/propagation.py:460-463).  Validated, then (faithfully) unused.
    assert absorbing_boundary is None or absorbing_boundary in _BOUNDARIES, (
        f"The absorbing_boundary must be None or in {_BOUNDARIES}."
    )


def transfer_propagate(field: Field, z, n, pad_width, cval: float = 0, absorbing_boundary=None,
                       absorbing_boundary_width: float = 0.65, kykx=(0.0, 0.0), shift_yx=(0.0, 0.0),
                       output_dx=None, output_shape=None, use_czt: bool = True,
                       mode: Literal["full", "same"] = "full", *, precision=None) -> Field:
    """Fresnel transfer propagation (functional/propagation.py:168-252)."""
    _check_mode(mode)
    _check_boundary(absorbing_boundary)
    if output_dx is not None or output_shape is not None:
        from .rescaled import rescaled_propagate

        return rescaled_propagate(field, nat.CX_KERNEL_TRANSFER, z, n, pad_width, kykx=kykx, shift_yx=shift_yx,
                                  output_dx=output_dx, output_shape=output_shape, use_czt=use_czt, mode=mode,
                                  cval=cval, precision=precision)
    zs, _ = _z_array(z)
    # transfer_propagate broadcasts z only when it has more than one entry
    zshape = (zs.size,) if np.asarray(z).size > 1 else ()
    u = _run_prop2d(field, nat.CX_KERNEL_TRANSFER, zs, zshape, n, pad_width, kykx=kykx, mode=mode,
                    precision=precision, cval=cval)
    out = shift_grid(field.replace(u=u), shift_yx)
    return out


def asm_propagate(field: Field, z, n, pad_width, cval: float = 0, absorbing_boundary=None,
                  absorbing_boundary_width: float = 0.65, kykx=(0.0, 0.0), remove_evanescent: bool = False,
                  bandlimit: bool = False, shift_yx=(0.0, 0.0), output_dx=None, output_shape=None,
                  use_czt: bool = True, mode: Literal["full", "same"] = "full", *, precision=None) -> Field:
    """Angular-spectrum propagation; ``remove_evanescent=True`` is the "exact"
    method (functional/propagation.py:255-352)."""
    _check_mode(mode)
    _check_boundary(absorbing_boundary)
    if output_dx is not None or output_shape is not None:
        from .rescaled import rescaled_propagate

        return rescaled_propagate(field, nat.CX_KERNEL_ASM, z, n, pad_width, kykx=kykx, shift_yx=shift_yx,
                                  output_dx=output_dx, output_shape=output_shape, use_czt=use_czt, mode=mode,
                                  remove_evanescent=remove_evanescent, bandlimit=bandlimit, cval=cval,
                                  precision=precision)
    zs, zshape = _z_array(z)
    u = _run_prop2d(field, nat.CX_KERNEL_ASM, zs, zshape, n, pad_width, kykx=kykx, shift_yx=shift_yx,
                    remove_evanescent=remove_evanescent, bandlimit=bandlimit, mode=mode, precision=precision,
                    cval=cval)
    return shift_grid(field.replace(u=u), shift_yx)


def _planar_propagator(field: Field, propagator):
    """Explicit propagator -> planar (HP, py, px) device tensor + plane index map."""
    torch = nat.torch_mod()
    H = propagator if isinstance(propagator, torch.Tensor) else torch.as_tensor(np.asarray(propagator))
    H = H.to(device=field.device, dtype=torch.complex64)
    ny, nx = field.spatial_shape
    W = field.n_wv
    if field.chromatic:
        if H.ndim >= 3 and H.shape[-1] in (1, W) and tuple(H.shape[-3:-1]) == (ny, nx):
            H = H.movedim(-1, -3)  # (..., wv, py, px)
            if H.shape[-3] == 1 and W > 1:
                H = H.expand(*H.shape[:-3], W, ny, nx)
        elif tuple(H.shape[-2:]) == (ny, nx):
            H = H.unsqueeze(-3).expand(*H.shape[:-2], W, ny, nx)
        else:
            raise ValueError(f"propagator shape {tuple(H.shape)} does not match field {field.shape}")
        hb = tuple(H.shape[:-3])
    else:
        if tuple(H.shape[-2:]) != (ny, nx):
            raise ValueError(f"propagator shape {tuple(H.shape)} does not match field {field.shape}")
        hb = tuple(H.shape[:-2])
    H = H.reshape(-1, ny, nx).contiguous()
    return H, hb


def kernel_propagate(field: Field, propagator, absorbing_boundary=None, absorbing_boundary_width: float = 0.65,
                     output_dx=None, output_shape=None, shift_yx=(0.0, 0.0), use_czt: bool = False,
                     *, precision=None) -> Field:
    """``ifft2(fft2(u) * propagator)`` (functional/propagation.py:355-394, FFT branch)."""
    _check_boundary(absorbing_boundary)
    if output_dx is not None or output_shape is not None or use_czt:
        raise NotImplementedError("kernel_propagate with an explicit propagator supports the FFT branch only; "
                                  "use asm_propagate/transfer_propagate with output_dx/output_shape")
    H, hb = _planar_propagator(field, propagator)
    W = field.n_wv
    B = field.batch_shape
    out_batch = np.broadcast_shapes(B, hb)
    nb_out = int(np.prod(out_batch)) if out_batch else 1
    nh = int(np.prod(hb)) if hb else 1
    hidx = np.broadcast_to(np.arange(nh).reshape(hb if hb else ()), out_batch).reshape(-1)
    h_index = np.repeat(hidx * W, W) + np.tile(np.arange(W), nb_out)
    # reuse the batch-broadcast plane planner with a pseudo z batch of hb
    zs = np.zeros(max(nh, 1))
    zshape = hb
    u = _run_prop2d(field, nat.CX_KERNEL_EXPLICIT, zs, zshape, 1.0, 0, mode="full", H=H, h_index=h_index,
                    precision=precision)
    return shift_grid(field.replace(u=u), shift_yx)


def _fill_propagator(field: Field, kernel: int, z, n, kykx, shift_yx=(0.0, 0.0), bandlimit=False,
                     remove_evanescent=False, precision=None, shape=None):
    """Propagator for ``field`` (or for a grid of ``shape`` with the field's spacing)."""
    torch = nat.torch_mod()
    prec = precision or config.get_precision()
    zs, zshape = _z_array(z)
    ny, nx = field.spatial_shape if shape is None else (int(shape[0]), int(shape[1]))
    W = field.n_wv
    # one plane per (z, wv): the propagator does not depend on the field batch
    planes, out_batch, _, nb_out = _plan_planes(field, zs, zshape, ny, nx, shift_yx, bandlimit, prec,
                                                batch_shape=())
    d = nat.cx_prop2d_desc()
    d.ny, d.nx, d.pad_y, d.pad_x = ny, nx, 0, 0
    d.n_wv = W
    d.n_in_planes = W
    d.n_out_planes = nb_out * W
    d.kernel = kernel
    d.precision = config.precision_code(prec)
    d.remove_evanescent = int(bool(remove_evanescent))
    d.bandlimit = int(bool(bandlimit))
    d.n_medium = float(n)
    ky0, kx0 = np.asarray(kykx, dtype=np.float64).reshape(2)
    d.ky0, d.kx0 = float(ky0), float(kx0)
    H = torch.empty((nb_out * W, ny, nx), dtype=torch.complex64, device=field.device)
    planes_dev = nat.to_device_bytes(planes, field.device)
    nat.check(nat.lib().cx_fill_propagator(d, nat.ptr(planes_dev), nat.ptr(H), nat.stream_handle(field.device)))
    H = H.reshape(tuple(out_batch) + (W, ny, nx))
    if field.chromatic:
        return H.movedim(-3, -1).contiguous()
    return H.reshape(tuple(out_batch) + (ny, nx))


def compute_transfer_propagator(field: Field, z, n, kykx=(0.0, 0.0), *, precision=None):
    """Fresnel transfer kernel, ifftshifted (functional/propagation.py:466-496)."""
    return _fill_propagator(field, nat.CX_KERNEL_TRANSFER, z, n, kykx, precision=precision)


def compute_asm_propagator(field: Field, z, n, kykx=(0.0, 0.0), bandlimit: bool = False, shift_yx=(0.0, 0.0),
                           remove_evanescent: bool = False, *, precision=None):
    """Angular-spectrum kernel, ifftshifted (functional/propagation.py:499-580)."""
    return _fill_propagator(field, nat.CX_KERNEL_ASM, z, n, kykx, shift_yx, bandlimit, remove_evanescent,
                            precision=precision)


def compute_padding_transform(height: int, wavelength: float, dx: float, z: float) -> int:
    """functional/propagation.py:583-605."""
    D = height * dx
    Nf = np.max((D / 2) ** 2 / (wavelength * z))
    M = height
    Q = 2 * np.maximum(1.0, M / (4 * Nf))
    N = (np.ceil((Q * M) / 2) * 2).astype(int)
    return int(N - M)


compute_padding_transfer = compute_padding_transform  # functional/propagation.py:608-630 (same rule)


def compute_padding_exact(height: int, wavelength: float, dx: float, z: float) -> int:
    """functional/propagation.py:633-656."""
    D = height * dx
    Nf = np.max((D / 2) ** 2 / (wavelength * z))
    M = height
    Q = 2 * np.maximum(1.0, M / (4 * Nf))
    scale = np.max((wavelength / (2 * dx)))
    Q = Q / np.sqrt(1 - scale**2)
    N = (np.ceil((Q * M) / 2) * 2).astype(int)
    return int(N - M)


def transform_propagate(field: Field, z, n, pad_width, cval: float = 0, skip_initial_phase: bool = False,
                        skip_final_phase: bool = False, *, precision=None) -> Field:
    """Single-FFT Fresnel propagation (functional/propagation.py:34-82)."""
    from .convenience import _optical_fft_chirped

    return _optical_fft_chirped(field, z, n, pad_width, cval, skip_initial_phase, skip_final_phase,
                                precision=precision)


def compute_sas_precompensation(field: Field, z, n, *, precision=None):
    """SAS precompensation Delta H of ``field``'s grid, ifftshifted
    (functional/propagation.py:85-103)."""
    return _fill_propagator(field, nat.CX_KERNEL_SAS, z, n, (0.0, 0.0), precision=precision)


def transform_propagate_sas(field: Field, z, n, cval: float = 0, skip_initial_phase: bool = False,
                            skip_final_phase: bool = False, *, precision=None) -> Field:
    """Scalable angular spectrum (functional/propagation.py:106-165): pad x2,
    precompensate with Delta H and take one transform step (z >= 0), or the
    transform step first and then Delta H of the transformed grid (z < 0);
    crop back.  Delta H is evaluated on the fly in the Fourier-multiplier
    pass (``CX_KERNEL_SAS``); the transform step is the chirped optical FFT,
    with the final crop fused into its store when z >= 0."""
    from .convenience import _dx_like, run_optfft
    from .sources import materialize

    if cval != 0:
        raise NotImplementedError("non-zero cval padding is not supported by the fused loader")
    field = materialize(field)
    z = float(np.asarray(z).reshape(()))
    sz = np.array(field.spatial_shape)
    pw = tuple(int(v) for v in sz // 2)
    c = np.pi / (field.spectrum.wavelength * z / float(n))
    chirps = dict(post=1j, chirp_in=None if skip_initial_phase else c, chirp_out=None if skip_final_phase else c,
                  precision=precision)
    if z >= 0:
        u1 = _run_prop2d(field, nat.CX_KERNEL_SAS, np.array([z]), (), n, pw, mode="full", precision=precision)
        f1 = field.replace(u=u1)
        u2, du = run_optfft(f1, z, float(n), pad_width=(0, 0), crop_width=pw, **chirps)
        return field.replace(u=u2, dx=_dx_like(f1, du))
    u1, du = run_optfft(field, z, float(n), pad_width=pw, crop_width=(0, 0), **chirps)
    f1 = field.replace(u=u1, dx=_dx_like(field, du))
    u2 = _run_prop2d(f1, nat.CX_KERNEL_SAS, np.array([z]), (), n, 0, mode="full", precision=precision)
    return crop(f1.replace(u=u2), pw)
