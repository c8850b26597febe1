"""Process-wide defaults.

``precision`` selects how phase arguments are evaluated by every kernel:

* ``"accurate"`` (default): FP64 phase arguments reduced mod 2 pi, FP32 FFT.
  Results sit within ~1e-6 relative L2 of an FP64 evaluation.
* ``"ref32"``: FP32 in the reference's operation order, reproducing the
  argument rounding of Chromatix's float32 JAX path (e.g. ~1.3e-4 relative
  L2 for angular-spectrum propagation at z = 100 um).
* ``"split16"``: as ``"accurate"``, with the column transforms of the passes
  that have a tensor-core form -- the PSF column pass and the Fourier-
  multiplier column pass of the propagators and the multislice slice loop,
  on padded grids of 1024 or 1280 rows (columns a multiple of 8) -- run as
  dense DFT contractions on FP16 hi + lo operands with FP32 accumulation
  (~2e-7 relative error per transform); every other pass runs as
  ``"accurate"``.
"""

from __future__ import annotations

import contextlib

_PRECISION = "accurate"
_VALID = ("accurate", "ref32", "split16")


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


def tensor_core_grid(py: int, px: int) -> bool:
    """Padded grids whose column transforms have a tensor-core form."""
    return py in (1024, 1280) and px % 8 == 0 and px >= 8


def precision_code(p: str | None = None, tensor_core: bool = False) -> int:
    """cx_precision of ``p`` for one entry point; ``tensor_core``: the entry
    point accepts CX_PREC_SPLIT16 (elsewhere "split16" means "accurate")."""
    p = p or _PRECISION
    if p not in _VALID:
        raise ValueError(f"precision must be one of {_VALID}, got {p!r}")
    if p == "split16":
        return 2 if tensor_core else 0
    return 0 if p == "accurate" else 1
