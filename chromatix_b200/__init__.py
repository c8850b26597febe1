"""chromatix_b200: B200-native (sm_100a) FFT-propagation hot path of Chromatix.

Same call signatures and Field semantics as ``chromatix.functional`` for the
propagation path; the compute runs in hand-written CUDA kernels behind the C
ABI of ``include/cx_b200.h`` (``chromatix_b200/_lib/libcx_b200.so``).
"""

from . import config
from .config import get_precision, precision, set_precision
from .core import ChromaticScalarField, ChromaticVectorField, Field, MonoSpectrum, ScalarField, Spectrum, VectorField, crop, pad, shift_grid

__all__ = ["Field", "ScalarField", "ChromaticScalarField", "VectorField", "ChromaticVectorField", "Spectrum", "MonoSpectrum", "pad", "crop", "shift_grid",
           "config", "set_precision", "get_precision", "precision", "functional"]


def __getattr__(name):
    if name == "functional":
        import importlib

        return importlib.import_module(".functional", __name__)
    raise AttributeError(name)
