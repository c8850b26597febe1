"""Ray-transfer (ABCD) propagation (functional/rays.py): the ABCD matrices of
free space and lenses, and Collins' integral through one native call
(``cx_ray_transfer``: an FP64 input chirp, the Fresnel transfer kernel of
z = B / M, an FP64 output chirp)."""

from __future__ import annotations

import numpy as np

from .. import _native as nat
from .. import config
from ..core.field import Field

__all__ = ["ray_transfer", "compute_free_space_abcd", "compute_thin_spherical_lens_abcd",
           "compute_plano_convex_spherical_lens_abcd"]


def compute_free_space_abcd(z) -> np.ndarray:
    """ABCD matrix of free space over ``z`` (functional/rays.py:14-28)."""
    return np.array([[1.0, float(z)], [0.0, 1.0]])


def compute_thin_spherical_lens_abcd(f, inverse: bool = False) -> np.ndarray:
    """ABCD matrix of a thin lens of focal length ``f`` (functional/rays.py:31-49)."""
    f = -float(f) if inverse else float(f)
    return np.array([[1.0, 0.0], [-1.0 / f, 1.0]])


def compute_plano_convex_spherical_lens_abcd(f, radius, center_thickness, n_lens, n_medium=1.0,
                                             inverse: bool = False) -> np.ndarray:
    """ABCD matrix of a thick plano-convex lens, exit @ centre @ entrance
    (functional/rays.py:52-99)."""
    center = np.array([[1.0, float(center_thickness)], [0.0, 1.0]])
    if inverse:
        entrance = np.array([[1.0, 0.0], [0.0, n_medium / n_lens]])
        exit_ = np.array([[1.0, 0.0], [(n_lens - n_medium) / (-radius * n_medium), n_lens / n_medium]])
    else:
        entrance = np.array([[1.0, 0.0], [(n_medium - n_lens) / (radius * n_lens), n_medium / n_lens]])
        exit_ = np.array([[1.0, 0.0], [0.0, n_lens / n_medium]])
    return exit_ @ center @ entrance


class cx_ray_desc(nat.ctypes.Structure):
    _fields_ = ([(k, nat.c_int32) for k in ("ny", "nx", "n_wv", "n_planes", "precision", "reserved")] +
                [(k, nat.ctypes.c_double) for k in ("A", "B", "D", "magnification", "n_medium", "origin_y",
                                                     "origin_x")])


def _lib():
    L = nat.lib()
    if not hasattr(L, "_cx_ray_sig"):
        P = nat.ctypes.POINTER(cx_ray_desc)
        L.cx_ray_transfer_workspace_size.restype = nat.c_int32
        L.cx_ray_transfer_workspace_size.argtypes = [P, nat.ctypes.POINTER(nat.c_size_t)]
        L.cx_ray_transfer.restype = nat.c_int32
        L.cx_ray_transfer.argtypes = [P, nat.c_void_p, nat.c_void_p, nat.c_void_p, nat.c_void_p, nat.c_size_t,
                                      nat.c_void_p]
        L._cx_ray_sig = True
    return L


def ray_transfer(field: Field, ABCD, n, magnification=1.0, *, precision=None) -> Field:
    """Collins' integral through the system ``ABCD`` (functional/rays.py:102-154):
    input chirp k (A - M) |g|^2 / (2B), centred FFT, exp(-i pi (lambda / n)
    (B / M) |f|^2), centred inverse FFT, output chirp
    k (D - 1/M) |g / M^2|^2 / (2B); the output spacing is dx / M."""
    from .propagation import _plan_planes
    from .sources import materialize

    torch = nat.torch_mod()
    nat.refuse_grad("ray_transfer", getattr(field, "u", None))
    field = materialize(field)
    if getattr(field, "vectorial", False):
        raise NotImplementedError("ray_transfer takes scalar fields")
    nat.require_cuda(field.u, "Field.u")
    M = np.asarray(ABCD, dtype=np.float64)
    ny, nx = field.spatial_shape
    planes, _, nb_in, _ = _plan_planes(field, np.zeros(1), (), ny, nx)
    W = field.n_wv
    org = np.asarray(field.origin, dtype=np.float64).reshape(-1, 2)[0]
    d = cx_ray_desc(ny=ny, nx=nx, n_wv=W, n_planes=nb_in * W, precision=config.precision_code(precision),
                    A=float(M[0, 0]), B=float(M[0, 1]), D=float(M[1, 1]), magnification=float(magnification),
                    n_medium=float(n), origin_y=float(org[0]), origin_x=float(org[1]))
    L = _lib()
    wsb = nat.c_size_t(0)
    nat.check(L.cx_ray_transfer_workspace_size(d, wsb))
    dev = field.device
    u = field.u.contiguous()
    out = torch.empty_like(u)
    ws = nat.workspace(wsb.value, dev)
    planes_dev = nat.to_device_bytes(planes, dev)
    nat.check(L.cx_ray_transfer(d, nat.ptr(planes_dev), nat.ptr(u), nat.ptr(out), nat.ptr(ws), wsb.value,
                                nat.stream_handle(dev)))
    return field.replace(u=out, dx=np.asarray(field.dx, dtype=np.float64) / float(magnification))
