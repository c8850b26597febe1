"""``fourier_convolution`` (ops/ops.py:9-86) on the GPU.

Real inputs convolved plane by plane over their last two axes
(``axes=(-2, -1)``), mode "same" -- the configuration the ``Microscope``
uses -- run as one native call (``cx_conv2d_same``): r2c row passes, column
passes with the product accumulated per plane, and the c2r back, all fused.
The kernel has its own plane shape and either the image's leading axes or
none (one 2D kernel for every plane).  ``reduce=True`` also sums over the
leading plane axes (``BasicSensor(reduce_axis=0)``) inside the same call.

Transform lengths: the reference pads to the next power of two of the summed
shape (``fast_fft_shape=True``) or to the summed shape itself; every length
>= 2 n - 1 gives the same linear convolution after the crop, so both settings
run at the smallest engine lengths >= 2 n (1536 -> 3072 instead of 4096).
``lengths="pow2"`` keeps the reference's power-of-two lengths.
"""

from __future__ import annotations

import numpy as np

from .. import _native as nat


class cx_conv_desc(nat.ctypes.Structure):
    _fields_ = [(k, nat.c_int32) for k in ("n_planes", "h", "w", "kh", "kw", "kernel_broadcast", "reduce",
                                           "pow2_lengths")]


def _lib():
    L = nat.lib()
    if not hasattr(L, "_cx_conv_sig"):
        P = nat.ctypes.POINTER(cx_conv_desc)
        L.cx_conv2d_workspace_size.restype = nat.c_int32
        L.cx_conv2d_workspace_size.argtypes = [P, nat.ctypes.POINTER(nat.c_size_t)]
        L.cx_conv2d_same.restype = nat.c_int32
        L.cx_conv2d_same.argtypes = [P, nat.c_void_p, nat.c_void_p, nat.c_void_p, nat.c_void_p, nat.c_size_t,
                                     nat.c_void_p]
        L._cx_conv_sig = True
    return L


def fourier_convolution(image, kernel, *, axes=(-2, -1), fast_fft_shape: bool = True, mode: str = "same",
                        reduce: bool = False, lengths: str = "smallest"):
    """Convolution ``kernel * image`` over the last two axes by the Fourier
    convolution theorem (ops/ops.py:9-86); ``reduce`` sums the result over
    all leading axes.  ``lengths``: "smallest" (smallest engine lengths
    >= 2 n) or "pow2" (next powers of two); the result is the same."""
    nat.refuse_grad("fourier_convolution", image, kernel)
    torch = nat.torch_mod()
    ax = tuple(a % image.ndim for a in axes)
    if ax != (image.ndim - 2, image.ndim - 1):
        raise NotImplementedError("convolution over the last two axes only")
    if mode != "same":
        raise NotImplementedError("mode='same' only")
    if lengths not in ("smallest", "pow2"):
        raise ValueError(f"lengths must be 'smallest' or 'pow2', got {lengths!r}")
    if image.ndim != kernel.ndim:
        raise AssertionError(f"Input ({image.ndim}D) and kernel ({kernel.ndim}D) must have same number of dimensions")
    if image.ndim < 2:
        raise NotImplementedError("convolution over two axes only")
    lead = tuple(image.shape[:-2])
    klead = tuple(kernel.shape[:-2])
    broadcast = all(k == 1 for k in klead)
    if klead != lead and not broadcast:
        raise NotImplementedError("the kernel's leading axes must equal the image's or be all 1")
    if torch.is_complex(image) or torch.is_complex(kernel):
        raise NotImplementedError("real inputs only (the rfftn branch)")
    nat.require_cuda(image, "image")
    a = image.to(torch.float32).contiguous()
    b = kernel.to(device=a.device, dtype=torch.float32).contiguous()
    h, w = a.shape[-2:]
    kh, kw = b.shape[-2:]
    planes = int(np.prod(lead)) if lead else 1
    d = cx_conv_desc(n_planes=planes, h=h, w=w, kh=kh, kw=kw, kernel_broadcast=1 if broadcast else 0,
                     reduce=1 if reduce else 0, pow2_lengths=1 if lengths == "pow2" else 0)
    L = _lib()
    wsb = nat.c_size_t(0)
    nat.check(L.cx_conv2d_workspace_size(d, wsb))
    ws = nat.workspace(wsb.value, a.device)
    out = torch.empty((h, w) if reduce else lead + (h, w), dtype=torch.float32, device=a.device)
    nat.check(L.cx_conv2d_same(d, nat.ptr(a), nat.ptr(b), nat.ptr(out), nat.ptr(ws), wsb.value,
                               nat.stream_handle(a.device)))
    return out
