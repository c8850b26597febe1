"""Utilities: chirp-Z transforms (reference: utils/czt.py)."""

from .czt import czt, cztn, zoomed_fft

__all__ = ["czt", "cztn", "zoomed_fft"]
