"""ctypes binding of the sm_100a shared library (``include/cx_b200.h``).

The library is the only compute path: if it is missing or cannot be loaded
every operation raises -- there is no CPU or eager fallback.  torch is used
for device memory, streams and host<->device copies only.
"""

from __future__ import annotations

import collections
import ctypes
import os
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libcx_b200.so")

c_double = ctypes.c_double
c_int32 = ctypes.c_int32
c_void_p = ctypes.c_void_p
c_size_t = ctypes.c_size_t

CX_OK = 0
CX_ERR_INVALID = 1
CX_ERR_UNSUPPORTED = 2
CX_ERR_CUDA = 3
CX_ERR_WORKSPACE = 4
CX_ERR_NOT_CONVERGED = 5
CX_PREC_ACCURATE = 0
CX_PREC_REF32 = 1
CX_KERNEL_TRANSFER = 0
CX_KERNEL_ASM = 1
CX_KERNEL_EXPLICIT = 2
CX_KERNEL_SAS = 3

_STATUS = {
    0: "CX_OK",
    1: "CX_ERR_INVALID",
    2: "CX_ERR_UNSUPPORTED",
    3: "CX_ERR_CUDA",
    4: "CX_ERR_WORKSPACE",
    5: "CX_ERR_NOT_CONVERGED",
}


class CxError(RuntimeError):
    """A non-zero ``cx_status`` from the native library."""

    def __init__(self, status: int, msg: str):
        super().__init__(f"{_STATUS.get(status, status)}: {msg}")
        self.status = status


class cx_plane(ctypes.Structure):
    _fields_ = [
        ("z", c_double),
        ("wavelength", c_double),
        ("dy", c_double),
        ("dx", c_double),
        ("shift_y", c_double),
        ("shift_x", c_double),
        ("bl_y0", c_double),
        ("bl_x0", c_double),
        ("bl_hy", c_double),
        ("bl_hx", c_double),
        ("in_plane", c_int32),
        ("h_plane", c_int32),
    ]


PLANE_DTYPE = np.dtype(
    [
        ("z", "<f8"),
        ("wavelength", "<f8"),
        ("dy", "<f8"),
        ("dx", "<f8"),
        ("shift_y", "<f8"),
        ("shift_x", "<f8"),
        ("bl_y0", "<f8"),
        ("bl_x0", "<f8"),
        ("bl_hy", "<f8"),
        ("bl_hx", "<f8"),
        ("in_plane", "<i4"),
        ("h_plane", "<i4"),
    ]
)
assert PLANE_DTYPE.itemsize == ctypes.sizeof(cx_plane)


class cx_prop2d_desc(ctypes.Structure):
    _fields_ = [
        ("ny", c_int32),
        ("nx", c_int32),
        ("pad_y", c_int32),
        ("pad_x", c_int32),
        ("n_wv", c_int32),
        ("n_in_planes", c_int32),
        ("n_out_planes", c_int32),
        ("mode_same", c_int32),
        ("kernel", c_int32),
        ("precision", c_int32),
        ("remove_evanescent", c_int32),
        ("bandlimit", c_int32),
        ("n_medium", c_double),
        ("ky0", c_double),
        ("kx0", c_double),
        ("conj_kernel", c_int32),
        ("crop_y", c_int32),
        ("crop_x", c_int32),
        ("reserved", c_int32),
    ]


class cx_ew_desc(ctypes.Structure):
    _fields_ = [
        ("n_batch", ctypes.c_int64),
        ("ny", c_int32),
        ("nx", c_int32),
        ("n_wv", c_int32),
        ("map_batched", c_int32),
    ]


class cx_psf_desc(ctypes.Structure):
    _fields_ = [
        ("ny", c_int32),
        ("nx", c_int32),
        ("n_z", c_int32),
        ("n_wv", c_int32),
        ("precision", c_int32),
        ("has_phase", c_int32),
        ("spectrally_modulate", c_int32),
        ("normalize_power", c_int32),
        ("f_obj", c_double),
        ("n_medium", c_double),
        ("NA", c_double),
        ("power", c_double),
        ("amplitude", c_double),
        ("offset_y", c_double),
        ("offset_x", c_double),
        ("f_lens", c_double),
        ("lens_NA", c_double),
    ]


class cx_psf_spectrum(ctypes.Structure):
    _fields_ = [
        ("wavelength", ctypes.POINTER(c_double)),
        ("density", ctypes.POINTER(c_double)),
        ("dy", ctypes.POINTER(c_double)),
        ("dx", ctypes.POINTER(c_double)),
    ]


# name -> (restype, argtypes)
_SIGS = {
    "cx_version": (c_int32, []),
    "cx_last_error": (ctypes.c_char_p, []),
    "cx_fft_size_supported": (c_int32, [c_int32]),
    "cx_fft1d": (c_int32, [c_void_p, c_void_p, c_int32, ctypes.c_int64, c_int32, c_void_p]),
    "cx_intensity": (c_int32, [c_void_p, ctypes.c_int64, c_int32, c_void_p, c_void_p, c_void_p]),
    "cx_prop2d_workspace_size": (c_int32, [ctypes.POINTER(cx_prop2d_desc), ctypes.POINTER(c_size_t)]),
    "cx_prop2d": (
        c_int32,
        [ctypes.POINTER(cx_prop2d_desc), c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_size_t, c_void_p],
    ),
    "cx_fill_propagator": (c_int32, [ctypes.POINTER(cx_prop2d_desc), c_void_p, c_void_p, c_void_p]),
    "cx_phase_change": (c_int32, [ctypes.POINTER(cx_ew_desc), c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "cx_phase_change_adjoint": (
        c_int32,
        [ctypes.POINTER(cx_ew_desc), c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p],
    ),
    "cx_thin_sample": (
        c_int32, [ctypes.POINTER(cx_ew_desc), c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]
    ),
    "cx_thin_sample_adjoint": (
        c_int32,
        [ctypes.POINTER(cx_ew_desc), c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
         c_void_p, c_void_p],
    ),
    "cx_intensity_adjoint": (c_int32, [c_void_p, ctypes.c_int64, c_int32, c_void_p, c_void_p, c_void_p, c_void_p]),
    "cx_pad": (
        c_int32,
        [ctypes.POINTER(cx_ew_desc), c_int32, c_int32, ctypes.c_float, ctypes.c_float, c_void_p, c_void_p, c_void_p],
    ),
    "cx_plane_wave": (
        c_int32,
        [ctypes.POINTER(cx_ew_desc), c_void_p, c_double, c_double, c_double, c_double, c_void_p, c_void_p],
    ),
    "cx_cmul_planar": (c_int32, [ctypes.POINTER(cx_ew_desc), c_void_p, c_void_p, c_int32, c_void_p, c_void_p]),
    "cx_pupil": (
        c_int32,
        [ctypes.POINTER(cx_ew_desc), c_int32, c_void_p, c_double, c_double, c_void_p, c_void_p, c_void_p],
    ),
    "cx_psf_workspace_size": (c_int32, [ctypes.POINTER(cx_psf_desc), ctypes.POINTER(c_size_t)]),
    "cx_psf_4f": (
        c_int32,
        [
            ctypes.POINTER(cx_psf_desc),
            ctypes.POINTER(cx_psf_spectrum),
            c_void_p,
            c_void_p,
            c_void_p,
            c_void_p,
            c_size_t,
            c_void_p,
        ],
    ),
}

_lib = None
_lock = threading.Lock()


def lib():
    """Load (once) and return the native library; raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"chromatix_b200 native library not found at {LIB_PATH}; "
                "build it with `python -m chromatix_b200.build` (no CPU fallback exists)"
            )
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != CX_OK:
        msg = lib().cx_last_error()
        raise CxError(status, msg.decode() if msg else "")


def exported_symbols():
    """Names declared in include/cx_b200.h that the loaded library must export."""
    return sorted(_SIGS)


# ---------------------------------------------------------------------------
# torch plumbing
# ---------------------------------------------------------------------------


def torch_mod():
    import torch

    return torch


def stream_handle(device=None) -> int:
    torch = torch_mod()
    return torch.cuda.current_stream(device).cuda_stream


def ptr(t) -> int:
    return 0 if t is None else int(t.data_ptr())


def workspace(nbytes: int, device):
    torch = torch_mod()
    return torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device)


def upload(arr: np.ndarray, device):
    """Host array -> device tensor through page-locked memory, asynchronous on
    the current stream: the host does not wait for the stream (a pageable
    blocking copy would synchronise it, serialising host and device)."""
    torch = torch_mod()
    t = torch.from_numpy(np.ascontiguousarray(arr)).pin_memory()
    return t.to(device, non_blocking=True)


# (descriptor type and bytes, plane table bytes, device) -> (workspace bytes,
# device plane table, event after its upload): repeated calls with the same
# geometry skip the workspace query and the host-to-device copy of their
# plane table.  The device tables are read-only; a call on another stream
# waits for the upload's event before its kernels read the table.
_TABLES = collections.OrderedDict()
_TABLES_SIZE = 128


def device_table(desc, planes: np.ndarray, device, ws_query):
    """(workspace bytes, device copy of ``planes``) for a launch described by
    the ctypes struct ``desc``; ``ws_query(desc)`` returns the workspace size."""
    torch = torch_mod()
    key = (type(desc).__name__, ctypes.string_at(ctypes.addressof(desc), ctypes.sizeof(desc)), planes.tobytes(),
           device.index)
    hit = _TABLES.get(key)
    if hit is not None:
        _TABLES.move_to_end(key)
        if not torch.cuda.is_current_stream_capturing():
            torch.cuda.current_stream(device).wait_event(hit[2])
        return hit[0], hit[1]
    ws_bytes = int(ws_query(desc))
    table = to_device_bytes(planes, device)
    ev = torch.cuda.Event()
    ev.record(torch.cuda.current_stream(device))
    _TABLES[key] = (ws_bytes, table, ev)
    if len(_TABLES) > _TABLES_SIZE:
        _TABLES.popitem(last=False)
    return ws_bytes, table


def to_device_bytes(arr: np.ndarray, device):
    """Copy a numpy (structured) array to device memory as raw bytes (asynchronously)."""
    return upload(np.ascontiguousarray(arr).view(np.uint8).reshape(-1), device)


_copy_streams = {}


def copy_stream(device):
    """A side stream per device for device-to-host result copies."""
    torch = torch_mod()
    dev = torch.device(device)
    idx = dev.index if dev.index is not None else torch.cuda.current_device()
    s = _copy_streams.get(idx)
    if s is None:
        s = _copy_streams[idx] = torch.cuda.Stream(device=idx)
    return s


def require_cuda(t, what="tensor"):
    if not t.is_cuda:
        raise ValueError(f"{what} must live on a CUDA device (the library has no CPU path)")


def wants_grad(*tensors) -> bool:
    """True when autograd is recording and one of ``tensors`` requires a gradient."""
    torch = torch_mod()
    return torch.is_grad_enabled() and any(isinstance(t, torch.Tensor) and t.requires_grad for t in tensors)


def refuse_grad(op: str, *tensors) -> None:
    """Raise instead of silently cutting the autograd graph: ``op`` writes its
    result through the native library and has no adjoint here."""
    if wants_grad(*tensors):
        raise NotImplementedError(
            f"{op}: no gradient is implemented for this operation (its result would be cut from the autograd "
            "graph); call it on detached inputs or under torch.no_grad()")
