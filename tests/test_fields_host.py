"""Host-side field logic without a GPU: Field.build's dispatch (scalar,
vector, chromatic), the vector field's layout (components innermost, spatial
axes -3, -2), padding and cropping of vector fields, and the 64-bit seed the
fluorescent sample derives from a key."""

import numpy as np
import pytest
import torch

import chromatix_b200 as cx
from chromatix_b200.core.field import crop, pad
from chromatix_b200.functional.samples import _seed_of


def test_build_dispatch_and_vector_layout():
    s = cx.Field.build(torch.zeros((8, 6), dtype=torch.complex64), 0.5, 0.5)
    v = cx.Field.build(torch.zeros((8, 6, 3), dtype=torch.complex64), 0.5, 0.5)
    c = cx.Field.build(torch.zeros((8, 6, 2), dtype=torch.complex64), 0.5, (np.array([0.5, 0.6]), np.ones(2)))
    assert type(s) is cx.ScalarField and type(v) is cx.VectorField and type(c) is cx.ChromaticScalarField
    assert v.spatial_dims == (-3, -2) and v.spatial_shape == (8, 6) and v.vectorial and not v.chromatic
    assert s.spatial_dims == (-2, -1) and not s.vectorial
    with pytest.raises(AssertionError):
        cx.VectorField(torch.zeros((8, 6, 2), dtype=torch.complex64), 0.5, 0.0, cx.MonoSpectrum(0.5))
    with pytest.raises(NotImplementedError):
        cx.Field.build(torch.zeros((2, 8, 6, 3), dtype=torch.complex64), 0.5, 0.5)


@pytest.mark.gpu
def test_pad_and_crop_vector_field():
    u = torch.arange(8 * 6 * 3, dtype=torch.float32).reshape(8, 6, 3).to(torch.complex64).cuda()
    v = cx.VectorField(u, 0.5, 0.0, cx.MonoSpectrum(0.5))
    p = pad(v, (2, 3))
    assert tuple(p.u.shape) == (12, 12, 3)
    assert torch.equal(p.u[2:10, 3:9], u) and p.u[0].abs().sum() == 0
    assert torch.equal(crop(p, (2, 3)).u, u)


def test_seed_of_key_forms():
    assert _seed_of(5) == 5
    assert _seed_of(np.array([1, 2], np.uint32)) == (1 << 32) | 2
    assert _seed_of(-1) == 0xFFFFFFFFFFFFFFFF


@pytest.mark.gpu
def test_chromatic_vector_field_layout_and_padding():
    wl = (np.array([0.5, 0.6]), np.ones(2))
    u = torch.arange(6 * 5 * 2 * 3, dtype=torch.float32).reshape(6, 5, 2, 3).to(torch.complex64).cuda()
    f = cx.Field.build(u, 0.4, wl)
    assert type(f) is cx.ChromaticVectorField and f.spatial_dims == (-4, -3) and f.spatial_shape == (6, 5)
    p = pad(f, (1, 2))
    assert tuple(p.u.shape) == (8, 9, 2, 3) and torch.equal(p.u[1:7, 2:7], u)
    assert torch.equal(crop(p, (1, 2)).u, u)


def test_pad_has_no_cpu_path():
    # the native pad kernel is the only implementation: a host tensor is refused
    u = torch.zeros((4, 4), dtype=torch.complex64)
    f = cx.Field.build(u, 0.5, 0.5)
    with pytest.raises(ValueError, match="CUDA"):
        pad(f, 1, 0.5)
