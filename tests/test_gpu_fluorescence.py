"""fluorescent_multislice_thick_sample (functional/samples.py:285-441) on the
GPU against the FP64 oracle: given phases and the library's phase generator
(bit-identical phases), several Monte-Carlo samples (the field carried from
one sample into the next, as in the reference), more slices than one
backward chunk, band limit / evanescent removal / tilt.
Tolerance: relative L2 <= 2e-5 (float32 transforms over D forward and D
backward slice steps)."""

import numpy as np
import pytest

from oracle import chromatix_oracle as O
from tests.helpers import rel, to_np

pytestmark = pytest.mark.gpu


def _inputs(shape, D, seed):
    rng = np.random.default_rng(seed)
    u = (rng.uniform(0.5, 1.0, shape) * np.exp(1j * rng.uniform(0, 0.3, shape))).astype(np.complex64)
    fl = rng.uniform(0, 1, (D,) + shape).astype(np.float32)
    dn = rng.uniform(-0.02, 0.02, (D,) + shape).astype(np.float32)
    return u, fl, dn


def _run(u, fl, dn, dx, lam, n, dz, pad, S, key=0, phases=None, **kw):
    import torch

    import chromatix_b200 as cx
    import chromatix_b200.functional as cf

    field = cx.Field.build(torch.as_tensor(u, device="cuda"), dx, lam)
    return to_np(cf.fluorescent_multislice_thick_sample(field, torch.as_tensor(fl, device="cuda"),
                                                        torch.as_tensor(dn, device="cuda"), n, dz, pad, key,
                                                        num_samples=S, random_phases=phases, **kw))


def _oracle(u, fl, dn, dx, lam, n, dz, pad, phases, **kw):
    f = O.field_build(u.astype(np.complex128), dx, lam)
    return O.fluorescent_multislice_thick_sample(f, fl.astype(np.float64), dn.astype(np.float64), n, dz, pad,
                                                 phases.astype(np.float64), **kw)


def test_given_phases_one_sample():
    shape, D = (48, 40), 6
    u, fl, dn = _inputs(shape, D, 0)
    ph = np.random.default_rng(1).uniform(0, 2 * np.pi, (1, D) + shape).astype(np.float32)
    out = _run(u, fl, dn, 0.3, 0.5, 1.33, 1.0, 8, 1, phases=ph)
    ref = _oracle(u, fl, dn, 0.3, 0.5, 1.33, 1.0, 8, ph)
    assert out.shape == (D,) + shape
    assert rel(out, ref) < 2e-5


def test_generated_phases_three_samples_carry_the_field():
    shape, D, S, seed = (32, 32), 4, 3, 1234567
    u, fl, dn = _inputs(shape, D, 2)
    ph = np.stack([O.fluor_phases(seed, s, (D,) + shape) for s in range(S)])
    out = _run(u, fl, dn, 0.4, 0.55, 1.0, 0.8, 16, S, key=seed)
    ref = _oracle(u, fl, dn, 0.4, 0.55, 1.0, 0.8, 16, ph)
    assert rel(out, ref) < 2e-5
    # the (2,) uint32 key form gives the same 64-bit seed
    out2 = _run(u, fl, dn, 0.4, 0.55, 1.0, 0.8, 16, S, key=np.array([seed >> 32, seed & 0xFFFFFFFF], np.uint32))
    np.testing.assert_array_equal(out, out2)


def test_more_slices_than_one_backward_chunk():
    shape, D = (24, 24), 40
    u, fl, dn = _inputs(shape, D, 3)
    ph = np.random.default_rng(4).uniform(0, 2 * np.pi, (1, D) + shape).astype(np.float32)
    out = _run(u, fl, dn, 0.5, 0.5, 1.2, 0.5, 4, 1, phases=ph)
    ref = _oracle(u, fl, dn, 0.5, 0.5, 1.2, 0.5, 4, ph)
    assert rel(out, ref) < 2e-5


def test_bandlimit_remove_evanescent_and_tilt():
    # dx = 0.15 um: the grid reaches evanescent frequencies, removed here
    shape, D = (40, 40), 5
    u, fl, dn = _inputs(shape, D, 5)
    ph = np.random.default_rng(6).uniform(0, 2 * np.pi, (2, D) + shape).astype(np.float32)
    kw = dict(kykx=(0.3, -0.2), remove_evanescent=True, bandlimit=True)
    out = _run(u, fl, dn, 0.15, 0.5, 1.33, 2.0, 12, 2, phases=ph, **kw)
    ref = _oracle(u, fl, dn, 0.15, 0.5, 1.33, 2.0, 12, ph, **kw)
    assert rel(out, ref) < 2e-5
