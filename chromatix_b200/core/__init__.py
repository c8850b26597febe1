"""Field and Spectrum containers (reference: core/field.py, core/spectrum.py)."""

from .field import ChromaticScalarField, ChromaticVectorField, Field, VectorField, ScalarField, crop, freq_grid, grid, pad, shift_grid
from .spectrum import MonoSpectrum, Spectrum

__all__ = ["Field", "ScalarField", "ChromaticScalarField", "VectorField", "ChromaticVectorField", "Spectrum", "MonoSpectrum", "pad", "crop",
           "shift_grid", "grid", "freq_grid"]
