"""Host logic of the batched propagation's L2 chunking: a batch whose planes
map one to one onto input planes is split into self-contained ranges of
fields whose intermediates fit L2_CHUNK_BYTES; z-broadcast batches (several
output planes per input) stay one call."""

import numpy as np

from chromatix_b200 import _native as nat
from chromatix_b200.functional import propagation as P


def _plan(n_fields, W, ny, nx, pad, in_plane=None, n_out=None, mode_same=0):
    d = nat.cx_prop2d_desc()
    d.ny, d.nx, d.pad_y, d.pad_x, d.n_wv = ny, nx, pad, pad, W
    d.n_in_planes = n_fields * W
    d.n_out_planes = n_out if n_out is not None else n_fields * W
    d.mode_same = mode_same
    planes = np.zeros(d.n_out_planes, dtype=nat.PLANE_DTYPE)
    planes["in_plane"] = np.arange(d.n_out_planes) if in_plane is None else in_plane
    return P._PropPlan(d, planes, (n_fields, ny, nx), (n_fields, ny + 2 * pad, nx + 2 * pad), W > 1)


def test_batch_of_64_fields_at_1024_splits_into_l2_sized_chunks():
    plan = _plan(64, 1, 512, 512, 256)
    per_field = 8 * 1024 * (512 + 1024)
    cf = P._chunk_fields(plan)
    assert cf == P.L2_CHUNK_BYTES // per_field == 5
    assert cf * per_field <= P.L2_CHUNK_BYTES


def test_small_batches_and_mode_same_fit_one_call():
    assert P._chunk_fields(_plan(4, 1, 512, 512, 256)) == 4
    # mode "same": the filtered spectra keep only the data rows
    plan = _plan(64, 3, 256, 256, 128, mode_same=1)
    per_field = 8 * 3 * 512 * (256 + 256)
    assert P._chunk_fields(plan) == min(64, P.L2_CHUNK_BYTES // per_field)


def test_z_broadcast_batches_are_not_split():
    # one field, 8 output planes reading input plane 0
    plan = _plan(1, 1, 1024, 1024, 512, in_plane=np.zeros(8, dtype=np.int32), n_out=8)
    assert P._chunk_fields(plan) == 1
    # two fields, each read by 4 planes
    plan = _plan(2, 1, 1024, 1024, 512, in_plane=np.repeat(np.arange(2), 4), n_out=8)
    assert P._chunk_fields(plan) == 2


def test_one_huge_field_is_one_chunk():
    assert P._chunk_fields(_plan(3, 1, 4096, 4096, 2048)) == 1
