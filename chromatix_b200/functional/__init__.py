"""Drop-in subset of ``chromatix.functional`` for the FFT-propagation hot path."""

from .convenience import optical_fft
from .lenses import df_lens, ff_lens, high_na_ff_lens, thin_lens
from .phase_masks import phase_change, spectrally_modulate_phase
from .propagation import (
    asm_propagate,
    compute_asm_propagator,
    compute_padding_exact,
    compute_padding_transfer,
    compute_padding_transform,
    compute_sas_precompensation,
    compute_transfer_propagator,
    kernel_propagate,
    transfer_propagate,
    transform_propagate,
    transform_propagate_sas,
)
from .rays import (
    compute_free_space_abcd,
    compute_plano_convex_spherical_lens_abcd,
    compute_thin_spherical_lens_abcd,
    ray_transfer,
)
from .pupils import circular_pupil, square_pupil, super_gaussian_pupil, tukey_pupil
from .samples import (
    fluorescent_multislice_thick_sample,
    multislice_thick_sample,
    polarized_multislice_thick_sample,
    thin_sample,
)
from .sources import objective_point_source, plane_wave
