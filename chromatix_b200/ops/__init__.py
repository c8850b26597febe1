"""Array operations of the imaging path (chromatix.ops subset)."""

from .convolution import fourier_convolution

__all__ = ["fourier_convolution"]
