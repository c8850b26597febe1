"""Process-wide defaults.

``precision`` selects how phase arguments are evaluated by every kernel:

* ``"accurate"`` (default): FP64 phase arguments reduced mod 2 pi, FP32 FFT.
  Results sit within ~1e-6 relative L2 of an FP64 evaluation.
* ``"ref32"``: FP32 in the reference's operation order, reproducing the
  argument rounding of Chromatix's float32 JAX path (e.g. ~1.3e-4 relative
  L2 for angular-spectrum propagation at z = 100 um).
"""

from __future__ import annotations

import contextlib

_PRECISION = "accurate"
_VALID = ("accurate", "ref32")


def get_precision() -> str:
    return _PRECISION


def set_precision(p: str) -> None:
    global _PRECISION
    if p not in _VALID:
        raise ValueError(f"precision must be one of {_VALID}, got {p!r}")
    _PRECISION = p


@contextlib.contextmanager
def precision(p: str):
    old = get_precision()
    set_precision(p)
    try:
        yield
    finally:
        set_precision(old)


def precision_code(p: str | None = None) -> int:
    p = p or _PRECISION
    if p not in _VALID:
        raise ValueError(f"precision must be one of {_VALID}, got {p!r}")
    return 0 if p == "accurate" else 1
