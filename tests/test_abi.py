"""The C-ABI library loads and exports every entry point include/*.h declares
(no compute: runs without a GPU)."""

import glob
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_ ]*[\s\*]+(cx_[A-Za-z0-9_]+)\s*\(", src, re.M):
            names.add(m.group(1))
    return sorted(names)


def _lib_path():
    from chromatix_b200 import _native as nat

    if not os.path.exists(nat.LIB_PATH):
        from chromatix_b200 import build

        build.build()
    return nat.LIB_PATH


def test_header_declares_entry_points():
    names = _declared()
    for n in ("cx_prop2d", "cx_psf_4f", "cx_optical_fft", "cx_last_error", "cx_fft1d"):
        assert n in names


def test_library_exports_every_declared_symbol():
    lib = _lib_path()
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True, check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if ln.strip()}
    missing = [n for n in _declared() if n not in exported]
    assert not missing, missing


def test_library_loads_without_gpu():
    from chromatix_b200 import _native as nat

    _lib_path()
    L = nat.lib()
    assert L.cx_version() >= 100
    assert L.cx_fft_size_supported(1280) == 1
    assert L.cx_fft_size_supported(143) == 0


def test_workspace_queries_and_validation_without_gpu():
    from chromatix_b200 import _native as nat

    _lib_path()
    L = nat.lib()
    d = nat.cx_prop2d_desc()
    d.ny, d.nx, d.pad_y, d.pad_x, d.n_wv, d.n_in_planes, d.n_out_planes = 512, 512, 256, 256, 1, 1, 1
    d.kernel, d.precision, d.n_medium = 1, 0, 1.33
    b = nat.c_size_t(0)
    assert L.cx_prop2d_workspace_size(d, b) == 0
    assert b.value >= 8 * (512 * 1024 + 1024 * 1024)
    d.ny = 0
    assert L.cx_prop2d_workspace_size(d, b) == 1
    assert b"invalid" in L.cx_last_error()
    d.ny, d.pad_y = 11, 0
    assert L.cx_prop2d_workspace_size(d, b) == 2  # 11 x 1024: length 11 not compiled in


def test_no_oracle_import_in_product():
    """The product package never imports the oracle."""
    for p in glob.glob(os.path.join(ROOT, "chromatix_b200", "**", "*.py"), recursive=True):
        src = open(p).read()
        assert "oracle" not in re.findall(r"^\s*(?:from|import)\s+(\S+)", src, re.M), p
