"""Incoherent imaging systems (systems/microscopes.py, elements/sensors.py).

``Microscope`` computes the PSF with its ``system_psf`` (an
``Optical4FSystemPSF``: objective point source -> phase mask -> tube lens,
the fused batched PSF pipeline), convolves it plane by plane with the sample
(``fourier_convolution`` over the last two axes) and hands the result to the
sensor.  A ``BasicSensor`` with ``reduce_axis=0`` sums the planes; that sum
runs inside the same native convolution call, so the per-plane images are
never materialised.  ``reduce_parallel_axis_name`` sums partial images over
the ranks of the default ``torch.distributed`` process group (the reference's
``psum`` over a pmapped axis).

Supported subset (what the reference's imaging benchmark uses): PSFs returned
as fields, ``padding_ratio = 0``, ``taper_width = 0``, no resampling, no shot
noise, 2D convolution over ``(-2, -1)`` of real samples of the PSF's shape.
"""

from __future__ import annotations

from typing import Any, Callable

import numpy as np

from . import _native as nat
from .core.spectrum import Spectrum
from .functional import ff_lens, objective_point_source, phase_change
from .ops import fourier_convolution

__all__ = ["Microscope", "Optical4FSystemPSF", "BasicSensor"]


class Optical4FSystemPSF:
    """PSF of a 4f system with a phase mask (systems/microscopes.py:300-365)."""

    def __init__(self, shape, spacing, f_tube, phase):
        self.shape = (int(shape[0]), int(shape[1]))
        self.spacing = spacing
        self.f_tube = f_tube
        self.phase = phase

    def __call__(self, microscope: "Microscope", z):
        if microscope.padding_ratio:
            raise NotImplementedError("padding_ratio > 0 is not part of this build")
        required = self.compute_required_spacing(self.shape[0], self.spacing, self.f_tube, microscope.n,
                                                 microscope.spectrum.wavelength)
        dx = required if microscope.spectrum.size > 1 else float(np.asarray(required).reshape(-1)[0])
        spec = (microscope.spectrum.wavelength, microscope.spectrum.density)
        field = objective_point_source(self.shape, dx, spec if microscope.spectrum.size > 1 else
                                       float(microscope.spectrum.wavelength[0]), z, microscope.f, microscope.n,
                                       microscope.NA, device=microscope.device)
        field = phase_change(field, self.phase)
        return ff_lens(field, self.f_tube, microscope.n)

    @staticmethod
    def compute_required_spacing(height, output_spacing, f, n, spectrum):
        return f * np.asarray(spectrum, dtype=np.float64) / (n * height * output_spacing)


class BasicSensor:
    """Intensity sensor (elements/sensors.py:14-118) without resampling or
    shot noise; ``reduce_axis`` sums the planes, ``reduce_parallel_axis_name``
    (any value) also sums over the ranks of the default process group."""

    def __init__(self, shape, spacing, shot_noise_mode=None, resampling_method="linear", reduce_axis=None,
                 reduce_parallel_axis_name=None):
        if shot_noise_mode is not None:
            raise NotImplementedError("shot noise is not part of this build")
        if resampling_method is not None:
            raise NotImplementedError("resampling is not part of this build (use resampling_method=None)")
        self.shape = tuple(shape)
        self.spacing = spacing
        self.shot_noise_mode = shot_noise_mode
        self.resampling_method = resampling_method
        self.reduce_axis = reduce_axis
        self.reduce_parallel_axis_name = reduce_parallel_axis_name

    def _parallel_sum(self, image):
        if self.reduce_parallel_axis_name is None:
            return image
        import torch.distributed as dist

        if dist.is_available() and dist.is_initialized():
            dist.all_reduce(image, op=dist.ReduceOp.SUM)
        return image

    def __call__(self, sensor_input, input_spacing=None, resample: bool = True, key=None):
        torch = nat.torch_mod()
        # a field's intensity is a computed property: read it once
        image = sensor_input if isinstance(sensor_input, torch.Tensor) else sensor_input.intensity
        if self.reduce_axis is not None:
            image = torch.sum(image, dim=self.reduce_axis)
        return self._parallel_sum(image)


class Microscope:
    """Microscope with a plane-wise spatially invariant PSF
    (systems/microscopes.py:16-297)."""

    def __init__(self, system_psf: Callable, sensor: BasicSensor, f, n, NA, spectrum, padding_ratio=0,
                 taper_width=0, convolution_axes=(-2, -1), fast_fft_shape: bool = True, *, device="cuda",
                 fft_lengths: str = "smallest"):
        if taper_width:
            raise NotImplementedError("taper_width > 0 is not part of this build")
        self.system_psf = system_psf
        self.sensor = sensor
        self.f, self.n, self.NA = f, n, NA
        self.spectrum = Spectrum.build(spectrum)
        self.padding_ratio = padding_ratio
        self.taper_width = taper_width
        self.convolution_axes = tuple(convolution_axes)
        self.fast_fft_shape = fast_fft_shape
        self.device = device
        # "smallest" engine lengths >= 2 n or "pow2" (the reference's
        # fast_fft_shape lengths): the same image either way
        self.fft_lengths = fft_lengths

    def psf(self, *args: Any, **kwargs: Any):
        return self.system_psf(self, *args, **kwargs)

    def __call__(self, sample, *args: Any, key=None, **kwargs: Any):
        torch = nat.torch_mod()
        system_psf = self.psf(*args, **kwargs)
        # the PSF field's intensity runs the fused PSF pipeline: evaluate it once
        psf = system_psf if isinstance(system_psf, torch.Tensor) else system_psf.intensity
        return self.image(sample, psf, key=key)

    def image(self, sample, psf, key=None):
        """fourier_convolution(sample, psf) over ``convolution_axes`` and the
        sensor (systems/microscopes.py:271-297)."""
        torch = nat.torch_mod()
        if not isinstance(sample, torch.Tensor):
            sample = torch.as_tensor(np.asarray(sample, np.float32), device=psf.device)
        sample = sample.to(device=psf.device)
        s = self.sensor
        fused = (s.reduce_axis == 0 and sample.ndim == 3 and s.shot_noise_mode is None
                 and s.resampling_method is None)
        if fused:
            image = fourier_convolution(sample, psf, axes=self.convolution_axes,
                                        fast_fft_shape=self.fast_fft_shape, reduce=True, lengths=self.fft_lengths)
            return s._parallel_sum(image)
        image = fourier_convolution(sample, psf, axes=self.convolution_axes, fast_fft_shape=self.fast_fft_shape,
                                    lengths=self.fft_lengths)
        return s(image, s.spacing, resample=False, key=key)
