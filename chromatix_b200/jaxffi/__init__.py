"""The jax.ffi route into the library (import-guarded: needs jax).

The reference is traced JAX code; a chromatix build that dispatches its
propagation hot path to this library registers the XLA FFI handler in
``cx_jax_ffi.cc`` as a CUDA custom-call target and calls it with
``jax.ffi.ffi_call``.  ``asm_propagate`` / ``transfer_propagate`` below are
that call for monochromatic (..., ny, nx) complex64 fields, with a
``jax.custom_vjp`` whose backward is the same handler with the conjugate
propagator (the adjoint; functional/propagation.py:391-394).

The handler library is compiled on first use from ``cx_jax_ffi.cc`` against
``jax.ffi.include_dir()`` and ``libcx_b200.so``; without jax, ``available()``
is False and nothing here runs.
"""

from __future__ import annotations

import ctypes
import functools
import os
import shutil
import subprocess

import numpy as np

from .. import _native as nat

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "cx_jax_ffi.cc")
LIB = os.path.join(os.path.dirname(nat.LIB_PATH), "libcx_jax_ffi.so")
INCLUDE = os.path.join(os.path.dirname(os.path.dirname(HERE)), "include")


def available() -> bool:
    """True when jax (with its FFI headers) can be imported."""
    try:
        import jax
        import jax.ffi  # noqa: F401
    except Exception:
        return False
    inc = getattr(jax.ffi, "include_dir", None)
    return inc is not None and os.path.isdir(inc())


def build(force: bool = False) -> str:
    """Compile the FFI handler library (needs jax's FFI headers and nvcc's host compiler)."""
    import jax.ffi

    if os.path.exists(LIB) and not force and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    cmd = [nvcc, "-std=c++17", "-O2", "-shared", "-Xcompiler", "-fPIC", "-x", "cu", SRC, "-I", jax.ffi.include_dir(),
           "-I", INCLUDE, "-L", os.path.dirname(nat.LIB_PATH), "-lcx_b200", "-Xlinker", "-rpath=$ORIGIN",
           "-o", LIB]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return LIB


@functools.lru_cache(maxsize=None)
def register() -> bool:
    """Register ``cx_prop2d`` as a CUDA custom-call target (once)."""
    import jax

    nat.lib()  # the C ABI library first (the handler library links against it)
    h = ctypes.CDLL(build())
    jax.ffi.register_ffi_target("cx_prop2d", jax.ffi.pycapsule(h.cx_prop2d_ffi), platform="CUDA")
    return True


def _desc_and_planes(shape, z, n, pad, dx, wavelength, kernel, mode, precision, conj, adjoint):
    """Descriptor attributes, plane table bytes, output shape and workspace
    bytes of one (forward or adjoint) propagation of a (..., ny, nx) field."""
    ny, nx = int(shape[-2]), int(shape[-1])
    batch = int(np.prod(shape[:-2])) if len(shape) > 2 else 1
    py, px = pad
    a = dict(ny=ny, nx=nx, pad_y=py, pad_x=px, crop_y=0, crop_x=0, mode_same=int(mode == "same"), kernel=kernel,
             precision=precision, remove_evanescent=0, bandlimit=0, conj_kernel=int(conj), n_medium=float(n),
             ky0=0.0, kx0=0.0)
    if adjoint and mode != "same":
        # the adjoint of a "full" propagation reads the padded grid (``shape`` is
        # the forward output's) without padding it and crops the padding off
        a.update(pad_y=0, pad_x=0, crop_y=py, crop_x=px)
    planes = np.zeros(batch, dtype=nat.PLANE_DTYPE)
    planes["z"] = float(z)
    planes["wavelength"] = float(wavelength)
    planes["dy"], planes["dx"] = float(dx[0]), float(dx[1])
    planes["in_plane"] = np.arange(batch)
    d = nat.cx_prop2d_desc(**{k: a[k] for k in ("ny", "nx", "pad_y", "pad_x", "mode_same", "kernel", "precision",
                                                  "remove_evanescent", "bandlimit", "n_medium", "ky0", "kx0",
                                                  "conj_kernel", "crop_y", "crop_x")},
                           n_wv=1, n_in_planes=batch, n_out_planes=batch)
    ws = nat.c_size_t(0)
    nat.check(nat.lib().cx_prop2d_workspace_size(d, ws))
    if a["mode_same"]:
        oy, ox = a["ny"], a["nx"]
    else:
        oy, ox = a["ny"] + 2 * a["pad_y"] - 2 * a["crop_y"], a["nx"] + 2 * a["pad_x"] - 2 * a["crop_x"]
    return a, planes.view(np.uint8), tuple(shape[:-2]) + (oy, ox), max(int(ws.value), 256)


def _ffi_prop(u, z, n, pad, dx, wavelength, kernel, mode, precision, conj, adjoint):
    import jax
    import jax.numpy as jnp

    attrs, planes, out_shape, ws = _desc_and_planes(u.shape, z, n, pad, dx, wavelength, kernel, mode, precision,
                                                    conj, adjoint)
    call = jax.ffi.ffi_call("cx_prop2d", (jax.ShapeDtypeStruct(out_shape, jnp.complex64),
                                          jax.ShapeDtypeStruct((ws,), jnp.uint8)))
    out, _ = call(u.astype(jnp.complex64), jnp.asarray(planes),
                  **{k: (np.int32(v) if isinstance(v, int) else np.float64(v)) for k, v in attrs.items()})
    return out


def _propagate(u, z, n, pad_width, dx, wavelength, kernel, mode, precision):
    import jax

    register()
    pad = (int(pad_width), int(pad_width)) if np.ndim(pad_width) == 0 else tuple(int(p) for p in pad_width)
    dxy = np.broadcast_to(np.asarray(dx, dtype=np.float64).reshape(-1), (2,))
    args = (float(z), float(n), pad, tuple(dxy), float(wavelength), kernel, mode, precision)

    @jax.custom_vjp
    def f(v):
        return _ffi_prop(v, *args, conj=False, adjoint=False)

    def fwd(v):
        return f(v), None

    def bwd(_, g):
        # jax's cotangent convention for complex outputs is the conjugate of
        # torch's: conj(A^H conj(g)) = A^T g
        gg = _ffi_prop(g.conj(), *args, conj=True, adjoint=True)
        return (gg.conj(),)

    f.defvjp(fwd, bwd)
    return f(u)


def asm_propagate(u, z, n, pad_width, dx, wavelength, mode="full", precision=nat.CX_PREC_ACCURATE):
    """``asm_propagate`` of a monochromatic (..., ny, nx) jax array through the
    library (functional/propagation.py:255-352, FFT branch)."""
    return _propagate(u, z, n, pad_width, dx, wavelength, nat.CX_KERNEL_ASM, mode, precision)


def transfer_propagate(u, z, n, pad_width, dx, wavelength, mode="full", precision=nat.CX_PREC_ACCURATE):
    """``transfer_propagate`` of a monochromatic (..., ny, nx) jax array through
    the library (functional/propagation.py:168-252, FFT branch)."""
    return _propagate(u, z, n, pad_width, dx, wavelength, nat.CX_KERNEL_TRANSFER, mode, precision)
