"""Shared test helpers: seeded inputs and CUDA <-> oracle conversions."""

import numpy as np

from oracle import chromatix_oracle as O


def rand_field(shape, seed=0, amp=(0.5, 1.0)):
    """``A exp(i phi)``, A ~ U[amp], phi ~ U[0, 2 pi) -- the synthetic field of
    the single-field ASM benchmark, complex64."""
    rng = np.random.default_rng(seed)
    a = rng.uniform(amp[0], amp[1], shape)
    ph = rng.uniform(0, 2 * np.pi, shape)
    return (a * np.exp(1j * ph)).astype(np.complex64)


def to_np(t):
    return t.detach().cpu().numpy()


def cuda_field(u, dx, spectrum):
    import torch

    import chromatix_b200 as cx

    return cx.Field.build(torch.as_tensor(u, device="cuda"), dx, spectrum)


def oracle_field(u, dx, spectrum, prec=O.FP64):
    return O.field_build(u, dx, spectrum, prec)


def rel(a, b):
    return O.rel_l2(a, b)
