"""cx_czt_noalloc (scratch in a static device buffer, no allocation) against
cx_czt (caller workspace) through the C ABI: identical outputs on two calls in
a row with different transforms, no change in free device memory once the
first call has done its set-up, and the size limit of the static scratch."""

import ctypes
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _lib():
    from chromatix_b200 import _native as nat

    czt_mod = importlib.import_module("chromatix_b200.utils.czt")
    L = czt_mod._lib()
    L.cx_czt_noalloc.restype = ctypes.c_int32
    L.cx_czt_noalloc.argtypes = [ctypes.POINTER(czt_mod.cx_czt_desc), ctypes.c_void_p, ctypes.c_void_p,
                                 ctypes.c_void_p]
    return nat, czt_mod, L


def _desc(czt_mod, shape, axis, m, a, w, scale=1.0, mod_n=-1):
    n = shape[axis]
    outer = int(np.prod(shape[:axis])) if axis > 0 else 1
    inner = int(np.prod(shape[axis + 1:])) if axis + 1 < len(shape) else 1
    d = czt_mod.cx_czt_desc()
    d.n, d.m, d.L, d.inner = n, m, 0, inner
    d.n_vec = outer * inner
    d.in_ostride, d.in_istride, d.in_estride = n * inner, 1, inner
    d.out_ostride, d.out_istride, d.out_estride = m * inner, 1, inner
    d.a_re, d.a_im, d.w_re, d.w_im = a.real, a.imag, w.real, w.imag
    d.mod_n, d.layout, d.scale = mod_n, 0 if inner == 1 else 1, scale
    oshape = list(shape)
    oshape[axis] = m
    return d, tuple(oshape)


def _both(nat, L, d, x, oshape):
    import torch

    y_ws = torch.empty(oshape, dtype=torch.complex64, device=x.device)
    y_na = torch.full(oshape, float("nan"), dtype=torch.complex64, device=x.device)
    b = nat.c_size_t(0)
    nat.check(L.cx_czt_workspace_size(d, b))
    ws = nat.workspace(b.value, x.device)
    st = nat.stream_handle(x.device)
    nat.check(L.cx_czt(d, nat.ptr(x), nat.ptr(y_ws), nat.ptr(ws), b.value, st))
    nat.check(L.cx_czt_noalloc(d, nat.ptr(x), nat.ptr(y_na), st))
    return y_ws, y_na


def test_noalloc_czt_matches_workspace_entry_point_two_calls_in_a_row():
    import torch

    nat, czt_mod, L = _lib()
    rng = np.random.default_rng(7)
    cases = [
        # rows, zoomed band (CZT branch of kernel_propagate), then columns with a different n / m / L
        ((3, 200), 1, 512, np.exp(1j * 0.3), np.exp(-1j * 2 * np.pi / 900), 1.0, -1),
        ((150, 96), 0, 90, np.exp(-1j * 0.7), np.exp(1j * 2 * np.pi / 400) * 1.0005, 0.25, 40),
    ]
    for rep in range(2):
        for shape, axis, m, a, w, scale, mod_n in cases:
            x = torch.as_tensor((rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64),
                                device="cuda")
            d, oshape = _desc(czt_mod, shape, axis, m, a, w, scale, mod_n)
            y_ws, y_na = _both(nat, L, d, x, oshape)
            torch.cuda.synchronize()
            assert torch.equal(y_ws, y_na), (rep, shape)


def test_noalloc_czt_allocates_no_device_memory():
    import torch

    nat, czt_mod, L = _lib()
    x = torch.ones((4, 256), dtype=torch.complex64, device="cuda")
    y = torch.empty((4, 300), dtype=torch.complex64, device="cuda")
    d, _ = _desc(czt_mod, (4, 256), 1, 300, 1.0 + 0j, np.exp(-1j * 2 * np.pi / 700))
    st = nat.stream_handle(x.device)
    nat.check(L.cx_czt_noalloc(d, nat.ptr(x), nat.ptr(y), st))  # set-up on first use
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    alloc0 = torch.cuda.memory_allocated()
    for _ in range(5):
        nat.check(L.cx_czt_noalloc(d, nat.ptr(x), nat.ptr(y), st))
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert torch.cuda.memory_allocated() == alloc0


def test_noalloc_czt_rejects_lengths_beyond_the_static_scratch():
    nat, czt_mod, L = _lib()
    d, _ = _desc(czt_mod, (1, 3000), 1, 2000, 1.0 + 0j, np.exp(-1j * 0.001))
    st = L.cx_czt_noalloc(d, None, None, None)
    assert st == 2
    assert b"static scratch" in L.cx_last_error()
