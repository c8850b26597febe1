"""Descriptor validation and workspace queries of the widened entry points,
through the C ABI without a GPU: invalid descriptors come back as
CX_ERR_INVALID / CX_ERR_UNSUPPORTED with a message, valid ones give the
documented workspace sizes."""

import ctypes

import pytest

from chromatix_b200 import _native as nat

CX_ERR_INVALID, CX_ERR_UNSUPPORTED = 1, 2


def _size(fn, d):
    n = ctypes.c_size_t(0)
    st = fn(ctypes.byref(d), ctypes.byref(n))
    return st, n.value, nat.lib().cx_last_error().decode()


def test_convolution_plan():
    from chromatix_b200.ops.convolution import _lib, cx_conv_desc

    L = _lib()
    st, n, _ = _size(L.cx_conv2d_workspace_size, cx_conv_desc(n_planes=2, h=1536, w=1536, kh=1536, kw=1536,
                                                              kernel_broadcast=0, reduce=1, pow2_lengths=0))
    assert st == 0 and n > 0
    st, _, msg = _size(L.cx_conv2d_workspace_size, cx_conv_desc(n_planes=1, h=3000, w=8, kh=3000, kw=8))
    assert st == CX_ERR_UNSUPPORTED and "longer than 4096" in msg
    st, _, _ = _size(L.cx_conv2d_workspace_size, cx_conv_desc(n_planes=0, h=8, w=8, kh=8, kw=8))
    assert st == CX_ERR_INVALID


def test_polarized_plan():
    from chromatix_b200.functional.samples import _polar_lib, cx_polar_desc

    L = _polar_lib()
    ok = dict(ny=256, nx=256, n_slices=4, n_wv=1, wv=0, n_medium=1.33, wavelength=0.55, dy=0.2, dx=0.2, dz=0.5,
              NA=1.0)
    st, n, _ = _size(L.cx_polarized_multislice_workspace_size, cx_polar_desc(**ok))
    # two x-spectrum buffers (N, 2M, 3), e U (2N, 2M, 3), the {e, h} table (2N, 2M)
    assert st == 0 and n >= 2 * 256 * 512 * 3 * 8 + 512 * 512 * 3 * 8 + 512 * 512 * 16
    st, _, msg = _size(L.cx_polarized_multislice_workspace_size, cx_polar_desc(**dict(ok, ny=255)))
    assert st == CX_ERR_INVALID and "even field sizes" in msg
    st, _, _ = _size(L.cx_polarized_multislice_workspace_size, cx_polar_desc(**dict(ok, wv=1)))
    assert st == CX_ERR_INVALID
    st, _, _ = _size(L.cx_polarized_multislice_workspace_size, cx_polar_desc(**dict(ok, ny=4096, nx=4096)))
    assert st == CX_ERR_UNSUPPORTED


def test_high_na_plan():
    from chromatix_b200.functional.lenses import _high_na_lib, cx_high_na_desc

    L = _high_na_lib()
    ok = dict(n_fields=1, ny=512, nx=512, my=256, mx=320, vectorial=1, f=100.0, n_medium=1.33, NA=0.8,
              wavelength=0.532, dy=0.3, dx=0.3, origin_y=0.0, origin_x=0.0, output_dx=0.1)
    st, n, _ = _size(L.cx_high_na_ff_lens_workspace_size, cx_high_na_desc(**ok))
    assert st == 0 and n >= (512 * 512 + 256 * 512) * 3 * 8
    for bad in (dict(my=1), dict(nx=1), dict(vectorial=2), dict(output_dx=0.0)):
        st, _, _ = _size(L.cx_high_na_ff_lens_workspace_size, cx_high_na_desc(**dict(ok, **bad)))
        assert st == CX_ERR_INVALID, bad


def test_ray_transfer_rejects_b_zero_without_gpu():
    from chromatix_b200.functional.rays import _lib, cx_ray_desc

    L = _lib()
    d = cx_ray_desc(ny=64, nx=64, n_wv=1, n_planes=1, precision=0, A=1.0, B=0.0, D=1.0, magnification=1.0,
                    n_medium=1.0)
    st, _, msg = _size(L.cx_ray_transfer_workspace_size, d)
    assert st == CX_ERR_INVALID and "B != 0" in msg
    d.B, d.n_planes, d.n_wv = 10.0, 3, 2  # planes not a multiple of the wavelengths
    st, _, _ = _size(L.cx_ray_transfer_workspace_size, d)
    assert st == CX_ERR_INVALID


def test_fluorescence_plan_rejects_bad_descriptors():
    from chromatix_b200.functional.samples import _fluor_lib, cx_fluor_desc

    L = _fluor_lib()
    d = cx_fluor_desc(ny=64, nx=64, pad=16, n_slices=4, num_samples=0, n_medium=1.0, wavelength=0.5, dy=0.3,
                      dx=0.3, dz=1.0)
    st, _, _ = _size(L.cx_fluorescent_multislice_workspace_size, d)
    assert st == CX_ERR_INVALID
    d.num_samples, d.pad = 1, 1  # 66: no FFT length
    st, _, msg = _size(L.cx_fluorescent_multislice_workspace_size, d)
    assert st == CX_ERR_UNSUPPORTED and "not supported" in msg
