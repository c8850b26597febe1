"""Spectrum: wavelengths and spectral density (core/spectrum.py:10-107).

Values are kept in float64 on the host: they are per-plane launch
parameters, not device arrays.  ``float32`` rounding of the reference is
reproduced by the ``"ref32"`` precision mode of the kernels.
"""

from __future__ import annotations

import dataclasses

import numpy as np


@dataclasses.dataclass(frozen=True, eq=False)
class Spectrum:
    wavelength: np.ndarray
    density: np.ndarray

    @property
    def size(self) -> int:
        return int(self.wavelength.size)

    @property
    def central_wavelength(self) -> float:
        """First wavelength of the spectrum (core/spectrum.py:75-83)."""
        return float(self.wavelength[0])

    @property
    def spectral_modulation(self) -> np.ndarray:
        """lambda0 / lambda (core/spectrum.py:88-90)."""
        return self.central_wavelength / self.wavelength

    @classmethod
    def build(cls, spectrum) -> "Spectrum":
        """``Spectrum.build`` (core/spectrum.py:37-73).

        float -> MonoSpectrum; (wavelengths, densities) -> Spectrum with the
        density normalised to sum 1; array of size 1 -> MonoSpectrum; other
        arrays -> Spectrum with equal densities.
        """
        if isinstance(spectrum, Spectrum):
            return spectrum
        if isinstance(spectrum, (float, int, np.floating, np.integer)):
            return MonoSpectrum(float(spectrum))
        if isinstance(spectrum, (tuple, list)):
            wl = np.atleast_1d(np.asarray(spectrum[0], dtype=np.float64))
            d = np.atleast_1d(np.asarray(spectrum[1], dtype=np.float64))
            if wl.ndim != 1:
                raise ValueError("Wavelength must be 1D for polychromatic spectrum.")
            if d.shape != wl.shape:
                raise ValueError(f"Density shape {d.shape} must match wavelength shape {wl.shape}.")
            return Spectrum(wl, d / d.sum())
        arr = np.asarray(spectrum, dtype=np.float64)
        if arr.size == 1:
            return MonoSpectrum(float(arr.reshape(())))
        if arr.ndim != 1:
            raise ValueError("Wavelength must be 1D for polychromatic spectrum.")
        return Spectrum(arr, np.full_like(arr, 1.0 / arr.size))


class MonoSpectrum(Spectrum):
    """Single wavelength (core/spectrum.py:96-107)."""

    def __init__(self, wavelength: float):
        wl = np.atleast_1d(np.asarray(wavelength, dtype=np.float64))
        if wl.shape != (1,):
            raise AssertionError(f"MonoSpectrum requires a scalar wavelength, got array of shape {wl.shape}")
        object.__setattr__(self, "wavelength", wl)
        object.__setattr__(self, "density", np.ones((1,)))
