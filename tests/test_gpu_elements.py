"""Element (module) API: each element equals the functional call it wraps,
and the reference's published PSF system composes into the fused pipeline."""

import numpy as np
import pytest

from oracle import chromatix_oracle as O
from tests.helpers import cuda_field, oracle_field, rand_field, rel, to_np

pytestmark = pytest.mark.gpu


def test_psf_optical_system_matches_functional_and_oracle():
    """examples/parallel_psf.py:20-27 at a small size."""
    import torch

    import chromatix_b200.functional as cf
    from chromatix_b200.elements import FFLens, ObjectivePointSource, OpticalSystem, PhaseMask

    shape, dx, lam, f, n, NA = (256, 256), 0.3, 0.532, 100.0, 1.33, 0.8
    z = np.linspace(-4, 4, 6)
    system = OpticalSystem([ObjectivePointSource(shape, dx, lam, f, n, NA), PhaseMask(np.ones(shape)), FFLens(f, n)])
    I = system(z).intensity
    ref = cf.ff_lens(cf.phase_change(cf.objective_point_source(shape, dx, lam, z, f, n, NA), np.ones(shape)), f, n)
    assert torch.equal(I, ref.intensity)
    o = O.ff_lens(O.phase_change(O.objective_point_source(shape, dx, lam, z, f, n, NA), np.ones(shape, np.float32)),
                  f, n)
    assert rel(to_np(I), o.intensity) < 1e-5


def test_propagate_elements():
    import torch

    import chromatix_b200.functional as cf
    from chromatix_b200.elements import KernelPropagate, Propagate

    u = rand_field((128, 128), seed=11)
    fc, fo = cuda_field(u, 0.3, 0.532), oracle_field(u, 0.3, 0.532)
    # default: cached band-limited ASM, mode "same"
    p = Propagate(fc, 50.0, 1.33, pad_width=64)
    out = p(fc)
    ref = O.asm_propagate(fo, 50.0, 1.33, 64, bandlimit=True, mode="same")
    assert out.u.shape == ref.u.shape
    assert rel(to_np(out.u), ref.u) < 1e-5
    for method in ("asm", "transfer"):
        q = Propagate(fc, 50.0, 1.33, pad_width=64, method=method, cache_propagator=False, bandlimit=False)
        fn = cf.asm_propagate if method == "asm" else cf.transfer_propagate
        assert torch.equal(q(fc).u, fn(fc, 50.0, 1.33, 64, mode="same").u)
    t = Propagate(fc, 50.0, 1.33, pad_width=64, method="transform", cache_propagator=False)
    assert torch.equal(t(fc).u, cf.transform_propagate(fc, 50.0, 1.33, 64).u)
    with pytest.raises(ValueError):
        Propagate(fc, 50.0, 1.33, method="transform")
    from chromatix_b200 import pad

    H = cf.compute_transfer_propagator(pad(fc, 64), 50.0, 1.33)
    k = KernelPropagate(H, pad_width=64)
    ref_t = O.transfer_propagate(fo, 50.0, 1.33, 64, mode="same")
    assert rel(to_np(k(fc).u), ref_t.u) < 1e-5


def test_multislice_element():
    import torch

    import chromatix_b200.functional as cf
    from chromatix_b200.elements import MultisliceThickSample

    rng = np.random.default_rng(2)
    dn = (0.02 * rng.standard_normal((6, 64, 64))).astype(np.float32)
    ab = rng.uniform(0, 0.05, (6, 64, 64)).astype(np.float32)
    fc = cuda_field(rand_field((64, 64), seed=1), 0.1, 0.532)
    s = MultisliceThickSample(ab, dn, 1.33, 0.1, 0.2, NA=0.8)
    assert s.num_planes == 6
    a = s(fc, pad_width=8)
    b = cf.multislice_thick_sample(fc, ab, dn, 1.33, 0.2, 8, NA=0.8)
    assert torch.equal(a.u, b.u)
    with pytest.raises(ValueError):
        MultisliceThickSample(ab, dn, 1.33, 0.2, 0.2)(fc)
