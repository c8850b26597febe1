"""Element (module) API of the propagation path: callables holding their
parameters, composed with :class:`OpticalSystem`.

Mirrors chromatix.elements (elements/propagation.py:20-228, lenses.py:11-171,
phase_masks.py:20-53, sources.py:193-510, samples.py:141-252) and
systems/optical_system.py:11-43, with the same constructor arguments and
defaults; each ``__call__`` is the functional call the reference makes.  The
fused paths are kept: ``OpticalSystem([ObjectivePointSource(...),
PhaseMask(...), FFLens(...)])(z).intensity`` runs the single batched PSF
pipeline, exactly like the functional composition.
"""

from __future__ import annotations

from typing import Any, Callable, Sequence

from . import functional as cf
from .core.field import Field, crop, pad

__all__ = ["Propagate", "KernelPropagate", "ThinLens", "FFLens", "DFLens", "PhaseMask", "ObjectivePointSource",
           "PlaneWave", "MultisliceThickSample", "OpticalSystem"]


class Propagate:
    """Free-space propagation by ``z`` (elements/propagation.py:20-178).

    Defaults as in the reference: ``method="asm"``, ``bandlimit=True``,
    ``mode="same"``, ``cache_propagator=True`` (the propagator of the padded
    ``field`` is computed once, here, and applied with ``kernel_propagate``).
    """

    def __init__(self, field: Field, z, n, pad_width: int = 0, cval: float = 0, kykx=(0.0, 0.0),
                 method: str = "asm", bandlimit: bool = True, remove_evanescent: bool = False, mode: str = "same",
                 cache_propagator: bool = True):
        self.z, self.n, self.pad_width, self.cval, self.kykx = z, n, pad_width, cval, kykx
        self.method, self.bandlimit, self.remove_evanescent = method, bandlimit, remove_evanescent
        self.mode, self.cache_propagator = mode, cache_propagator
        self.propagator = None
        if cache_propagator:
            padded = pad(field, pad_width, cval=cval)
            if method == "transfer":
                self.propagator = cf.compute_transfer_propagator(padded, z, n, kykx)
            elif method == "asm":
                self.propagator = cf.compute_asm_propagator(padded, z, n, kykx, bandlimit=bandlimit,
                                                            remove_evanescent=remove_evanescent)
            else:
                raise ValueError("Can only cache kernel for 'transfer' or 'asm' methods")

    def __call__(self, field: Field) -> Field:
        if self.cache_propagator:
            field = pad(field, self.pad_width, cval=self.cval)
            field = cf.kernel_propagate(field, self.propagator)
            if self.mode == "same":
                field = crop(field, self.pad_width)
            return field
        if self.method == "transform":
            return cf.transform_propagate(field, self.z, self.n, pad_width=self.pad_width, cval=self.cval)
        if self.method == "transfer":
            return cf.transfer_propagate(field, self.z, self.n, pad_width=self.pad_width, cval=self.cval,
                                         kykx=self.kykx, mode=self.mode)
        if self.method == "asm":
            return cf.asm_propagate(field, self.z, self.n, pad_width=self.pad_width, cval=self.cval, kykx=self.kykx,
                                    mode=self.mode, remove_evanescent=self.remove_evanescent,
                                    bandlimit=self.bandlimit)
        raise ValueError("Method must be one of: 'transform', 'transfer', 'asm'")


class KernelPropagate:
    """Propagation with a precomputed kernel (elements/propagation.py:181-228)."""

    def __init__(self, propagator, pad_width: int = 0, cval: float = 0.0, mode: str = "same"):
        self.propagator, self.pad_width, self.cval, self.mode = propagator, pad_width, cval, mode

    def __call__(self, field: Field) -> Field:
        field = pad(field, self.pad_width, cval=self.cval)
        field = cf.kernel_propagate(field, self.propagator)
        if self.mode == "same":
            field = crop(field, self.pad_width)
        return field


class ThinLens:
    """elements/lenses.py:11-51."""

    def __init__(self, f, n, NA=None):
        self.f, self.n, self.NA = f, n, NA

    def __call__(self, field: Field) -> Field:
        return cf.thin_lens(field, self.f, self.n, self.NA)


class FFLens:
    """elements/lenses.py:54-108."""

    def __init__(self, f, n, NA=None, inverse: bool = False):
        self.f, self.n, self.NA, self.inverse = f, n, NA, inverse

    def __call__(self, field: Field) -> Field:
        return cf.ff_lens(field, self.f, self.n, self.NA, inverse=self.inverse)


class DFLens:
    """elements/lenses.py:111-171."""

    def __init__(self, d, f, n, NA=None, inverse: bool = False):
        self.d, self.f, self.n, self.NA, self.inverse = d, f, n, NA, inverse

    def __call__(self, field: Field) -> Field:
        return cf.df_lens(field, self.d, self.f, self.n, self.NA, inverse=self.inverse)


class PhaseMask:
    """``field * exp(1j * phase)`` (elements/phase_masks.py:20-53)."""

    def __init__(self, phase):
        self.phase = phase

    def __call__(self, field: Field) -> Field:
        return cf.phase_change(field, self.phase)


class ObjectivePointSource:
    """Defocused point source behind an objective (elements/sources.py:193-357);
    called with ``z``."""

    def __init__(self, shape, dx, spectrum, f, n, NA, power=1.0, amplitude=1.0, offset=(0.0, 0.0),
                 scalar: bool = True, *, device="cuda"):
        self.shape, self.dx, self.spectrum = shape, dx, spectrum
        self.f, self.n, self.NA = f, n, NA
        self.power, self.amplitude, self.offset, self.scalar = power, amplitude, offset, scalar
        self.device = device

    def __call__(self, z) -> Field:
        return cf.objective_point_source(self.shape, self.dx, self.spectrum, z, self.f, self.n, self.NA, self.power,
                                         self.amplitude, self.offset, self.scalar, device=self.device)


class PlaneWave:
    """elements/sources.py:360-510."""

    def __init__(self, shape, dx, spectrum, power=1.0, amplitude=1.0, kykx=(0.0, 0.0), pupil=None,
                 scalar: bool = True, *, device="cuda"):
        self.shape, self.dx, self.spectrum = shape, dx, spectrum
        self.power, self.amplitude, self.kykx, self.pupil, self.scalar = power, amplitude, kykx, pupil, scalar
        self.device = device

    def __call__(self) -> Field:
        return cf.plane_wave(self.shape, self.dx, self.spectrum, self.power, self.amplitude, self.kykx, self.pupil,
                             self.scalar, device=self.device)


class MultisliceThickSample:
    """Thick sample as thin slices (elements/samples.py:141-252)."""

    def __init__(self, absorption, dn, n, dx, thickness, NA=None):
        self.absorption, self.dn, self.n, self.dx, self.thickness, self.NA = absorption, dn, n, dx, thickness, NA

    @property
    def shape(self):
        return tuple(self.absorption.shape)

    @property
    def num_planes(self) -> int:
        return int(self.absorption.shape[0])

    def __call__(self, field: Field, kykx=(0.0, 0.0), pad_width: int = 0, reverse_propagate_distance=None,
                 return_stack: bool = False, remove_evanescent: bool = False, bandlimit: bool = False) -> Field:
        import numpy as np

        if not np.allclose(np.asarray(field.dx, dtype=np.float64).reshape(-1),
                           np.broadcast_to(np.asarray(self.dx, dtype=np.float64), np.shape(field.dx)).reshape(-1)):
            raise ValueError("the sample's spacing does not match the field's")
        return cf.multislice_thick_sample(field, self.absorption, self.dn, self.n, self.thickness, pad_width,
                                          NA=self.NA, kykx=kykx, reverse_propagate_distance=reverse_propagate_distance,
                                          return_stack=return_stack, remove_evanescent=remove_evanescent,
                                          bandlimit=bandlimit)


class OpticalSystem:
    """A sequence of elements called in turn (systems/optical_system.py:11-43):
    the first element receives the call's arguments, each later one the
    previous element's field."""

    def __init__(self, elements: Sequence[Callable]):
        self.elements = list(elements)

    def __call__(self, *args: Any, **kwargs: Any):
        field = self.elements[0](*args, **kwargs)
        for element in self.elements[1:]:
            field = element(field)
        return field
