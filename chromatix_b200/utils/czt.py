"""Chirp-Z transforms on CUDA tensors (utils/czt.py:7-124).

``czt`` runs the fused Bluestein kernel of ``cx_czt`` along any axis without
moving data: a contiguous axis uses one team per vector, a strided axis is
processed in coalesced column tiles.  Chirp phases are evaluated in FP64
(the reference warns that its complex64 CZT is inaccurate: utils/czt.py:17-18).
"""

from __future__ import annotations

import numpy as np

from .. import _native as nat

__all__ = ["czt", "cztn", "zoomed_fft"]


class cx_czt_desc(nat.ctypes.Structure):
    _fields_ = [("n", nat.c_int32), ("m", nat.c_int32), ("L", nat.c_int32), ("inner", nat.c_int32),
                ("n_vec", nat.ctypes.c_int64), ("in_ostride", nat.ctypes.c_int64),
                ("in_istride", nat.ctypes.c_int64), ("in_estride", nat.ctypes.c_int64),
                ("out_ostride", nat.ctypes.c_int64), ("out_istride", nat.ctypes.c_int64),
                ("out_estride", nat.ctypes.c_int64), ("a_re", nat.c_double), ("a_im", nat.c_double),
                ("w_re", nat.c_double), ("w_im", nat.c_double), ("mod_n", nat.c_int32), ("layout", nat.c_int32),
                ("scale", nat.c_double), ("adjoint", nat.c_int32), ("reserved", nat.c_int32)]


_SIG = False


def _lib():
    global _SIG
    L = nat.lib()
    if not _SIG:
        P = nat.ctypes.POINTER(cx_czt_desc)
        L.cx_czt_workspace_size.restype = nat.c_int32
        L.cx_czt_workspace_size.argtypes = [P, nat.ctypes.POINTER(nat.c_size_t)]
        L.cx_czt.restype = nat.c_int32
        L.cx_czt.argtypes = [P, nat.c_void_p, nat.c_void_p, nat.c_void_p, nat.c_size_t, nat.c_void_p]
        _SIG = True
    return L


def _launch_czt(d: cx_czt_desc, x, oshape, out=None):
    torch = nat.torch_mod()
    y = out if out is not None else torch.empty(oshape, dtype=torch.complex64, device=x.device)
    L = _lib()
    ws_b = nat.c_size_t(0)
    nat.check(L.cx_czt_workspace_size(d, ws_b))
    ws = nat.workspace(ws_b.value, x.device)
    nat.check(L.cx_czt(d, nat.ptr(x), nat.ptr(y), nat.ptr(ws), ws_b.value, nat.stream_handle(x.device)))
    return y


def _adjoint_desc(d: cx_czt_desc) -> cx_czt_desc:
    """The transform's conjugate transpose: m inputs onto n outputs (the
    strides of input and output swap roles)."""
    a = cx_czt_desc.from_buffer_copy(d)
    a.adjoint = 1 - d.adjoint
    a.in_ostride, a.in_istride, a.in_estride = d.out_ostride, d.out_istride, d.out_estride
    a.out_ostride, a.out_istride, a.out_estride = d.in_ostride, d.in_istride, d.in_estride
    return a


_CZT_FN = None


def _czt_fn():
    """torch autograd Function over ``cx_czt``: the backward is the adjoint
    chirp-Z transform (``adjoint = 1``), one fused Bluestein pass like the
    forward (the gradient jax.grad takes through utils/czt.py:7-52)."""
    global _CZT_FN
    if _CZT_FN is None:
        torch = nat.torch_mod()

        class _CZT(torch.autograd.Function):
            @staticmethod
            def forward(ctx, x, d_bytes, oshape):
                ctx.d_bytes, ctx.ishape = d_bytes, tuple(x.shape)
                return _launch_czt(cx_czt_desc.from_buffer_copy(d_bytes), x, oshape)

            @staticmethod
            def backward(ctx, g):
                d = _adjoint_desc(cx_czt_desc.from_buffer_copy(ctx.d_bytes))
                return _launch_czt(d, g.to(torch.complex64).contiguous(), ctx.ishape), None, None

        _CZT_FN = _CZT
    return _CZT_FN


def czt_axis(x, m: int, a: complex, w: complex, axis: int = -1, mod_n: int = -1, scale: float = 1.0, out=None):
    """Low-level fused CZT of a contiguous complex64 CUDA tensor along ``axis``."""
    torch = nat.torch_mod()
    nat.require_cuda(x, "x")
    x = x.to(torch.complex64).contiguous()
    axis = axis % x.ndim
    n = x.shape[axis]
    outer = int(np.prod(x.shape[:axis])) if axis > 0 else 1
    inner = int(np.prod(x.shape[axis + 1:])) if axis + 1 < x.ndim else 1
    oshape = list(x.shape)
    oshape[axis] = m
    d = cx_czt_desc()
    d.n, d.m, d.L, d.inner = n, int(m), 0, inner
    d.n_vec = outer * inner
    d.in_ostride, d.in_istride, d.in_estride = n * inner, 1, inner
    d.out_ostride, d.out_istride, d.out_estride = m * inner, 1, inner
    a = complex(a)
    w = complex(w)
    d.a_re, d.a_im, d.w_re, d.w_im = a.real, a.imag, w.real, w.imag
    d.mod_n = int(mod_n)
    d.layout = 0 if inner == 1 else 1
    d.scale = float(scale)
    if nat.wants_grad(x):
        if out is not None:
            raise ValueError("czt_axis: out= is not differentiable")
        return _czt_fn().apply(x, bytes(d), tuple(oshape))
    return _launch_czt(d, x, tuple(oshape), out)


def czt(x, m: int, a, w, axis: int = -1):
    """Chirp-Z transform along one axis (utils/czt.py:7-52):
    ``y[k] = sum_j x[j] a^(-j) w^(j k)``, ``k < m``."""
    torch = nat.torch_mod()
    if not isinstance(x, torch.Tensor):
        x = torch.as_tensor(np.asarray(x), device="cuda")
    return czt_axis(x, m, complex(a), complex(w), axis)


def cztn(x, m, a, w, axes=(-2, -1)):
    """CZT along several axes in turn (utils/czt.py:55-80)."""
    for d, ax in enumerate(axes):
        x = czt(x, m[d], a[d], w[d], axis=ax)
    return x


def zoomed_fft(x, k_start: float, k_end: float, output_shape, axes=(-2, -1), include_end: bool = True):
    """Zoomed FFT over [k_start, k_end] via CZT (utils/czt.py:83-124)."""
    renorm = tuple(mm - 1 for mm in output_shape) if include_end else tuple(output_shape)
    w = tuple(np.exp(1j * (k_end - k_start) / nn) for nn in renorm)
    a = np.exp(-1j * k_start)
    return cztn(x, output_shape, tuple(a for _ in output_shape), w, axes)
