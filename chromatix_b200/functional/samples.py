"""Thin and thick samples (functional/samples.py:85-282)."""

from __future__ import annotations

import numpy as np

from .. import _native as nat
from ..core.field import Field

__all__ = ["thin_sample", "multislice_thick_sample", "fluorescent_multislice_thick_sample",
           "polarized_multislice_thick_sample"]


_THIN_FN = None


def _thin_fn():
    """autograd Function of ``cx_thin_sample``; the backward is
    ``cx_thin_sample_adjoint`` (gradients of the field, absorption and dn)."""
    global _THIN_FN
    if _THIN_FN is None:
        torch = nat.torch_mod()

        class _ThinSample(torch.autograd.Function):
            @staticmethod
            def forward(ctx, u, ab, dn, kd, d_bytes):
                d = nat.cx_ew_desc.from_buffer_copy(d_bytes)
                out = torch.empty_like(u)
                nat.check(nat.lib().cx_thin_sample(d, nat.ptr(u), nat.ptr(ab), nat.ptr(dn), nat.ptr(kd),
                                                   nat.ptr(out), nat.stream_handle(u.device)))
                ctx.d_bytes = d_bytes
                ctx.save_for_backward(out, ab, dn, kd)
                return out

            @staticmethod
            def backward(ctx, g):
                out, ab, dn, kd = ctx.saved_tensors
                d = nat.cx_ew_desc.from_buffer_copy(ctx.d_bytes)
                g = g.to(torch.complex64).contiguous()
                nu, na, nd = ctx.needs_input_grad[:3]
                gu = torch.empty_like(g) if nu else None
                ga = torch.empty_like(ab) if na else None
                gd = torch.empty_like(dn) if nd else None
                nat.check(nat.lib().cx_thin_sample_adjoint(d, nat.ptr(g), nat.ptr(out), nat.ptr(ab), nat.ptr(dn),
                                                           nat.ptr(kd), nat.ptr(gu), nat.ptr(ga), nat.ptr(gd),
                                                           nat.stream_handle(g.device)))
                return gu, ga, gd, None, None

        _THIN_FN = _ThinSample
    return _THIN_FN


def thin_sample(field: Field, absorption, dn, thickness) -> Field:
    """``u * exp(1j 2 pi (dn + 1j absorption) thickness / lambda)``
    (functional/samples.py:85-134), one pass of the native kernel
    ``cx_thin_sample``.  Inside ``multislice_thick_sample`` this product is
    fused into the slice kernel."""
    from .phase_masks import _ew_desc, channel_scale
    from .sources import materialize

    torch = nat.torch_mod()
    field = materialize(field)
    nat.require_cuda(field.u, "Field.u")
    ny, nx = field.spatial_shape

    def _map(m, what):
        t = m if isinstance(m, torch.Tensor) else torch.as_tensor(np.asarray(m, dtype=np.float32))
        if t.ndim != 2:
            raise AssertionError(f"{what} must have shape {field.spatial_shape}, got {tuple(t.shape)}")
        if tuple(t.shape) != (ny, nx):
            raise AssertionError(f"{what} must have shape {field.spatial_shape}, got {tuple(t.shape)}")
        return t.to(device=field.device, dtype=torch.float32).contiguous()

    a = _map(absorption, "Absorption")
    d_ = _map(dn, "Refractive index")
    kd = torch.as_tensor(channel_scale(field, 2 * np.pi * float(thickness) / field.spectrum.wavelength),
                         device=field.device)
    u = field.u.to(torch.complex64).contiguous()
    d = _ew_desc(field, 0)
    if nat.wants_grad(u, a, d_):
        out = _thin_fn().apply(u, a, d_, kd, bytes(d))
    else:
        out = torch.empty_like(u)
        nat.check(nat.lib().cx_thin_sample(d, nat.ptr(u), nat.ptr(a), nat.ptr(d_), nat.ptr(kd), nat.ptr(out),
                                           nat.stream_handle(u.device)))
    return field.replace(u=out)


class cx_ms_desc(nat.ctypes.Structure):
    _fields_ = [("ny", nat.c_int32), ("nx", nat.c_int32), ("pad", nat.c_int32), ("n_slices", nat.c_int32),
                ("precision", nat.c_int32), ("remove_evanescent", nat.c_int32), ("bandlimit", nat.c_int32),
                ("checkpoint_every", nat.c_int32), ("n_medium", nat.c_double), ("wavelength", nat.c_double),
                ("dy", nat.c_double), ("dx", nat.c_double), ("dz", nat.c_double),
                ("reverse_distance", nat.c_double), ("NA", nat.c_double), ("ky0", nat.c_double),
                ("kx0", nat.c_double)]


_MS_SIG = False


def _ms_lib():
    global _MS_SIG
    L = nat.lib()
    if not _MS_SIG:
        P = nat.ctypes.POINTER(cx_ms_desc)
        V = nat.c_void_p
        L.cx_multislice_workspace_size.restype = nat.c_int32
        L.cx_multislice_workspace_size.argtypes = [P, nat.c_int32, nat.ctypes.POINTER(nat.c_size_t)]
        L.cx_multislice_num_checkpoints.restype = nat.c_int32
        L.cx_multislice_num_checkpoints.argtypes = [P]
        L.cx_multislice_forward.restype = nat.c_int32
        L.cx_multislice_forward.argtypes = [P, V, V, V, V, V, V, nat.c_size_t, V]
        L.cx_multislice_backward.restype = nat.c_int32
        L.cx_multislice_backward.argtypes = [P, V, V, V, V, V, V, V, V, nat.c_size_t, V]
        _MS_SIG = True
    return L


def _ms_forward(d: cx_ms_desc, u, dn, ab, want_ckpt: bool):
    torch = nat.torch_mod()
    L = _ms_lib()
    dev = u.device
    ws_b = nat.c_size_t(0)
    nat.check(L.cx_multislice_workspace_size(d, 0, ws_b))
    ws = nat.workspace(ws_b.value, dev)
    out = torch.empty((d.ny, d.nx), dtype=torch.complex64, device=dev)
    ck = None
    if want_ckpt:
        nck = L.cx_multislice_num_checkpoints(d)
        ck = torch.empty((nck, d.ny + 2 * d.pad, d.nx + 2 * d.pad), dtype=torch.complex64, device=dev)
    nat.check(L.cx_multislice_forward(d, nat.ptr(u), nat.ptr(dn), nat.ptr(ab), nat.ptr(out), nat.ptr(ck),
                                      nat.ptr(ws), ws_b.value, nat.stream_handle(dev)))
    return out, ck


def _ms_backward(d: cx_ms_desc, dn, ab, ck, grad_out, need_u: bool):
    torch = nat.torch_mod()
    L = _ms_lib()
    dev = grad_out.device
    ws_b = nat.c_size_t(0)
    nat.check(L.cx_multislice_workspace_size(d, 1, ws_b))
    ws = nat.workspace(ws_b.value, dev)
    gdn = torch.empty_like(dn)
    gab = torch.empty_like(ab)
    gu = torch.empty((d.ny, d.nx), dtype=torch.complex64, device=dev) if need_u else None
    g = grad_out.to(torch.complex64).contiguous()
    nat.check(L.cx_multislice_backward(d, nat.ptr(dn), nat.ptr(ab), nat.ptr(ck), nat.ptr(g), nat.ptr(gdn),
                                       nat.ptr(gab), nat.ptr(gu), nat.ptr(ws), ws_b.value, nat.stream_handle(dev)))
    return gdn, gab, gu


def _autograd_fn():
    torch = nat.torch_mod()

    class _Multislice(torch.autograd.Function):
        """Forward: the fused multislice loop; backward: the hand-written adjoint
        (checkpoints every K slices, recomputation in between)."""

        @staticmethod
        def forward(ctx, u, dn, ab, desc_bytes):
            d = cx_ms_desc.from_buffer_copy(desc_bytes)
            need = ctx.needs_input_grad
            out, ck = _ms_forward(d, u.contiguous(), dn, ab, want_ckpt=any(need[:3]))
            ctx.desc_bytes = desc_bytes
            if any(need[:3]):
                ctx.save_for_backward(dn, ab, ck)
            return out

        @staticmethod
        def backward(ctx, grad_out):
            dn, ab, ck = ctx.saved_tensors
            d = cx_ms_desc.from_buffer_copy(ctx.desc_bytes)
            need = ctx.needs_input_grad
            gdn, gab, gu = _ms_backward(d, dn, ab, ck, grad_out, need_u=need[0])
            return (gu if need[0] else None, gdn if need[1] else None, gab if need[2] else None, None)

    return _Multislice


_MS_FN = None


def _multislice_stack(field: Field, absorption_stack, dn_stack, n, thickness_per_slice, pad_width, kykx,
                      remove_evanescent, bandlimit, precision) -> Field:
    """``return_stack=True`` (functional/samples.py:253-260): the field after
    every slice, without the final defocus, cropped; the plane index becomes
    the innermost batch axis.  Each slice is one call of the fused slice loop
    on the padded grid (differentiable like the whole stack)."""
    from ..core.field import crop, pad

    torch = nat.torch_mod()
    dn = dn_stack if isinstance(dn_stack, torch.Tensor) else torch.as_tensor(np.asarray(dn_stack, np.float32))
    ab = absorption_stack if isinstance(absorption_stack, torch.Tensor) else torch.as_tensor(
        np.asarray(absorption_stack, np.float32))
    dn = dn.to(device=field.device, dtype=torch.float32)
    ab = ab.to(device=field.device, dtype=torch.float32)
    if tuple(dn.shape) != tuple(ab.shape):
        raise AssertionError("absorption_stack and dn_stack must have equal shapes")
    p = int(pad_width)
    # center_pad of the stacks (samples.py:224-225): zero index change and absorption in the padding
    dn = torch.nn.functional.pad(dn, (p, p, p, p))
    ab = torch.nn.functional.pad(ab, (p, p, p, p))
    f = pad(field, p)
    planes = []
    for i in range(dn.shape[0]):
        f = multislice_thick_sample(f, ab[i:i + 1], dn[i:i + 1], n, thickness_per_slice, 0, kykx=kykx,
                                    reverse_propagate_distance=0.0, remove_evanescent=remove_evanescent,
                                    bandlimit=bandlimit, precision=precision)
        planes.append(f.u)
    axis = -4 if field.chromatic else -3
    return crop(field.replace(u=torch.stack(planes, dim=planes[0].ndim + axis + 1)), p)


def multislice_thick_sample(field: Field, absorption_stack, dn_stack, n, thickness_per_slice, pad_width: int,
                            NA=None, propagator=None, kykx=(0.0, 0.0), reverse_propagate_distance=None,
                            return_stack: bool = False, remove_evanescent: bool = False, bandlimit: bool = False,
                            *, checkpoint_every: int = 0, precision=None) -> Field:
    """Thick sample as D thin slices (functional/samples.py:137-282).

    Each slice: ``u <- t_i * IFFT2(H(dz) FFT2(u))`` with the ASM kernel H and
    ``t_i = exp(i 2 pi (dn_i + i abs_i) dz / lambda)``; afterwards the field is
    propagated back by ``reverse_propagate_distance`` (default: half the stack)
    with an optional NA mask, and cropped by ``pad_width``.  Differentiable with
    respect to the field, ``dn_stack`` and ``absorption_stack`` through a
    hand-written adjoint that stores a checkpoint every ``checkpoint_every``
    slices (default ceil(sqrt(D))) and recomputes in between.
    """
    from .. import config
    from .sources import materialize

    global _MS_FN
    torch = nat.torch_mod()
    field = materialize(field)
    if field.chromatic and field.n_wv != 1:
        raise NotImplementedError("multislice supports monochromatic scalar fields")
    if propagator is not None:
        raise NotImplementedError("a custom propagator is not supported by the fused slice kernel")
    if return_stack:
        return _multislice_stack(field, absorption_stack, dn_stack, n, thickness_per_slice, pad_width, kykx,
                                 remove_evanescent, bandlimit, precision)
    dev = field.device
    dn = dn_stack if isinstance(dn_stack, torch.Tensor) else torch.as_tensor(np.asarray(dn_stack, np.float32))
    ab = absorption_stack if isinstance(absorption_stack, torch.Tensor) else torch.as_tensor(
        np.asarray(absorption_stack, np.float32))
    dn = dn.to(device=dev, dtype=torch.float32).contiguous()
    ab = ab.to(device=dev, dtype=torch.float32).contiguous()
    if tuple(dn.shape) != tuple(ab.shape):
        raise AssertionError("absorption_stack and dn_stack must have equal shapes")
    D, ny, nx = dn.shape
    if (ny, nx) != tuple(field.spatial_shape):
        raise AssertionError("stack slices must match the field's spatial shape")
    if reverse_propagate_distance is None:
        reverse_propagate_distance = thickness_per_slice * D / 2
    d = cx_ms_desc()
    d.ny, d.nx, d.pad, d.n_slices = ny, nx, int(pad_width), D
    pp = (ny + 2 * int(pad_width), nx + 2 * int(pad_width))
    d.precision = config.precision_code(precision, tensor_core=config.tensor_core_grid(*pp))
    d.remove_evanescent, d.bandlimit = int(bool(remove_evanescent)), int(bool(bandlimit))
    d.checkpoint_every = int(checkpoint_every)
    d.n_medium = float(n)
    d.wavelength = float(field.spectrum.wavelength[0])
    d.dy, d.dx = (float(v) for v in field.dx_wv[0])
    d.dz = float(thickness_per_slice)
    d.reverse_distance = float(reverse_propagate_distance)
    d.NA = -1.0 if NA is None else float(NA)
    d.ky0, d.kx0 = (float(v) for v in np.asarray(kykx, np.float64).reshape(2))
    desc_bytes = bytes(d)
    if _MS_FN is None:
        _MS_FN = _autograd_fn()
    u = field.u
    lead = u.shape[:-3] if field.chromatic else u.shape[:-2]
    u2 = u.reshape((-1, ny, nx))
    outs = [_MS_FN.apply(u2[b], dn, ab, desc_bytes) for b in range(u2.shape[0])]
    out = torch.stack(outs).reshape(u.shape)
    return field.replace(u=out)


class cx_fluor_desc(nat.ctypes.Structure):
    _fields_ = ([(k, nat.c_int32) for k in ("ny", "nx", "pad", "n_slices", "num_samples", "remove_evanescent",
                                            "bandlimit", "reserved")] +
                [("seed", nat.ctypes.c_uint64)] +
                [(k, nat.c_double) for k in ("n_medium", "wavelength", "dy", "dx", "dz", "ky0", "kx0")])


def _fluor_lib():
    L = nat.lib()
    if not hasattr(L, "_cx_fluor_sig"):
        P = nat.ctypes.POINTER(cx_fluor_desc)
        V = nat.c_void_p
        L.cx_fluorescent_multislice_workspace_size.restype = nat.c_int32
        L.cx_fluorescent_multislice_workspace_size.argtypes = [P, nat.ctypes.POINTER(nat.c_size_t)]
        L.cx_fluorescent_multislice.restype = nat.c_int32
        L.cx_fluorescent_multislice.argtypes = [P, V, V, V, V, V, V, nat.c_size_t, V]
        L._cx_fluor_sig = True
    return L


def _seed_of(key) -> int:
    """64-bit generator seed from an int or a (2,) uint32 key (jax's PRNGKey data)."""
    k = np.asarray(key)
    if k.ndim == 0:
        return int(k) & 0xFFFFFFFFFFFFFFFF
    seed = 0
    for v in k.astype(np.uint64).reshape(-1):
        seed = ((seed << 32) ^ int(v)) & 0xFFFFFFFFFFFFFFFF
    return seed


def fluorescent_multislice_thick_sample(field: Field, fluorescence_stack, dn_stack, n, thickness_per_slice,
                                        pad_width: int, key, num_samples: int = 1, propagator_forward=None,
                                        propagator_backward=None, kykx=(0.0, 0.0), remove_evanescent: bool = False,
                                        bandlimit: bool = False, *, random_phases=None):
    """Thick, transparent, fluorescent sample (functional/samples.py:285-441):
    Monte-Carlo samples of random fluorophore phases; per sample the padded
    field goes through the slices (phase exp(i 2 pi dn dz / lambda), plus the
    fluorescence with its random phase, then an ASM step of ``dz``), and the
    stack of intensities comes from propagating the result back slice by slice.
    Returns the (D, h, w) float32 intensity stack averaged over the samples.

    One native call (``cx_fluorescent_multislice``).  Phases: ``random_phases``
    ((num_samples, D, h, w) radians) if given, else the library's counter-based
    generator seeded by ``key`` (an int or a (2,) uint32 key); the reference's
    jax.random stream is not reproduced.  As in the reference, each sample
    starts from the field the previous one ended with."""
    nat.refuse_grad("fluorescent_multislice_thick_sample", getattr(field, "u", None), fluorescence_stack, dn_stack)
    from .sources import materialize

    torch = nat.torch_mod()
    field = materialize(field)
    if field.chromatic or getattr(field, "vectorial", False):
        raise NotImplementedError("fluorescent multislice takes a monochromatic scalar field")
    if propagator_forward is not None or propagator_backward is not None:
        raise NotImplementedError("custom propagators are not supported by the fused slice kernels")
    dev = field.device
    fl = fluorescence_stack if isinstance(fluorescence_stack, torch.Tensor) else torch.as_tensor(
        np.asarray(fluorescence_stack, np.float32))
    dn = dn_stack if isinstance(dn_stack, torch.Tensor) else torch.as_tensor(np.asarray(dn_stack, np.float32))
    fl = fl.to(device=dev, dtype=torch.float32).contiguous()
    dn = dn.to(device=dev, dtype=torch.float32).contiguous()
    if tuple(fl.shape) != tuple(dn.shape):
        raise AssertionError("fluorescence_stack and dn_stack must have equal shapes")
    D, ny, nx = dn.shape
    if (ny, nx) != tuple(field.spatial_shape) or field.u.ndim != 2:
        raise AssertionError("one (h, w) field with stack slices of its shape is expected")
    S = int(num_samples)
    ph = None
    if random_phases is not None:
        ph = random_phases if isinstance(random_phases, torch.Tensor) else torch.as_tensor(
            np.asarray(random_phases, np.float32))
        ph = ph.to(device=dev, dtype=torch.float32).contiguous()
        if tuple(ph.shape) != (S, D, ny, nx):
            raise AssertionError(f"random_phases must have shape {(S, D, ny, nx)}, got {tuple(ph.shape)}")
    d = cx_fluor_desc()
    d.ny, d.nx, d.pad, d.n_slices, d.num_samples = ny, nx, int(pad_width), D, S
    d.remove_evanescent, d.bandlimit = int(bool(remove_evanescent)), int(bool(bandlimit))
    d.seed = _seed_of(key)
    d.n_medium = float(n)
    d.wavelength = float(field.spectrum.wavelength[0])
    d.dy, d.dx = (float(v) for v in field.dx_wv[0])
    d.dz = float(thickness_per_slice)
    d.ky0, d.kx0 = (float(v) for v in np.asarray(kykx, np.float64).reshape(2))
    L = _fluor_lib()
    wsb = nat.c_size_t(0)
    nat.check(L.cx_fluorescent_multislice_workspace_size(d, wsb))
    ws = nat.workspace(wsb.value, dev)
    u = field.u.contiguous()
    out = torch.empty((D, ny, nx), dtype=torch.float32, device=dev)
    nat.check(L.cx_fluorescent_multislice(d, nat.ptr(u), nat.ptr(fl), nat.ptr(dn),
                                          nat.ptr(ph) if ph is not None else None, nat.ptr(out), nat.ptr(ws),
                                          wsb.value, nat.stream_handle(dev)))
    return out


class cx_polar_desc(nat.ctypes.Structure):
    _fields_ = ([(k, nat.c_int32) for k in ("ny", "nx", "n_slices", "n_wv", "wv", "reserved")] +
                [(k, nat.c_double) for k in ("n_medium", "wavelength", "dy", "dx", "dz", "NA")])


def _polar_lib():
    L = nat.lib()
    if not hasattr(L, "_cx_polar_sig"):
        P = nat.ctypes.POINTER(cx_polar_desc)
        V = nat.c_void_p
        L.cx_polarized_multislice_workspace_size.restype = nat.c_int32
        L.cx_polarized_multislice_workspace_size.argtypes = [P, nat.ctypes.POINTER(nat.c_size_t)]
        L.cx_polarized_multislice.restype = nat.c_int32
        L.cx_polarized_multislice.argtypes = [P, V, V, V, V, nat.c_size_t, V]
        L._cx_polar_sig = True
    return L


def polarized_multislice_thick_sample(field: Field, potential_stack, n, thickness_per_slice, NA=1.0) -> Field:
    """Birefringent thick sample (functional/samples.py:444-546): a
    ``VectorField`` (or, wavelength by wavelength with the potential shared as
    in the reference, a ``ChromaticVectorField``) through the (D, h, w, 3, 3) scattering
    potential, per slice u <- P_op(u) + H_op(V_i Q_op(u)) with the vectorial
    free-space and scattering operators on the grid zero-padded to twice the
    size, band-limited to ``NA``.  One native call
    (``cx_polarized_multislice``): per slice two row passes and two column
    passes whose CTAs hold the three components, so the 3x3 k-space projector
    and the potential apply between the transforms."""
    nat.refuse_grad("polarized_multislice_thick_sample", getattr(field, "u", None), potential_stack)
    from .sources import materialize

    torch = nat.torch_mod()
    field = materialize(field)
    if not getattr(field, "vectorial", False):
        raise AssertionError("Must be a vectorial Field")
    nat.require_cuda(field.u, "Field.u")
    W = field.spectrum.size if field.chromatic else 1
    if field.u.ndim != (4 if field.chromatic else 3):
        raise NotImplementedError("one (h, w, 3) or (h, w, wv, 3) vector field")
    ny, nx = field.spatial_shape
    V = potential_stack if isinstance(potential_stack, torch.Tensor) else torch.as_tensor(
        np.asarray(potential_stack, np.float32))
    if torch.is_complex(V):
        raise NotImplementedError("real scattering potentials (the reference's Float array)")
    V = V.to(device=field.device, dtype=torch.float32).contiguous()
    if V.ndim != 5 or tuple(V.shape[1:]) != (ny, nx, 3, 3):
        raise AssertionError(f"potential_stack must have shape (D, {ny}, {nx}, 3, 3), got {tuple(V.shape)}")
    L = _polar_lib()
    u = field.u.contiguous()
    out = torch.empty_like(u)
    for w in range(W):  # independent wavelengths, one workspace in stream order
        d = cx_polar_desc(ny=ny, nx=nx, n_slices=V.shape[0], n_wv=W, wv=w, n_medium=float(n),
                          wavelength=float(field.spectrum.wavelength[w]), dz=float(thickness_per_slice), NA=float(NA))
        d.dy, d.dx = (float(v) for v in field.dx_wv[w])
        wsb = nat.c_size_t(0)
        nat.check(L.cx_polarized_multislice_workspace_size(d, wsb))
        ws = nat.workspace(wsb.value, field.device)
        nat.check(L.cx_polarized_multislice(d, nat.ptr(u), nat.ptr(V), nat.ptr(out), nat.ptr(ws), wsb.value,
                                            nat.stream_handle(field.device)))
    return field.replace(u=out)
