"""Host logic of the propagation plane tables: the vectorised construction in
functional/propagation.py equals a plane-by-plane restatement for batched,
chromatic, z-broadcast and explicit-propagator (h_index) cases."""

import types

import numpy as np
import pytest

from chromatix_b200 import _native as nat
from chromatix_b200.functional import propagation as P


def _stub(batch, W, dx, wl):
    return types.SimpleNamespace(batch_shape=tuple(batch), n_wv=W,
                                 dx_wv=np.broadcast_to(np.asarray(dx, np.float64).reshape(-1, 2), (W, 2)).copy(),
                                 spectrum=types.SimpleNamespace(wavelength=np.asarray(wl, np.float64).reshape(W)))


def _loop_planes(field, zs, zshape, shift_yx, h_index):
    B = field.batch_shape
    out_batch = np.broadcast_shapes(B, zshape)
    nb_in = int(np.prod(B)) if B else 1
    nb_out = int(np.prod(out_batch)) if out_batch else 1
    in_idx = np.broadcast_to(np.arange(nb_in).reshape(B if B else ()), out_batch).reshape(-1)
    z_idx = (np.broadcast_to(np.arange(zs.size).reshape(zshape), out_batch).reshape(-1) if zshape
             else np.zeros(nb_out, dtype=np.int64))
    W = field.n_wv
    planes = np.zeros(nb_out * W, dtype=nat.PLANE_DTYPE)
    for ob in range(nb_out):
        for w in range(W):
            q = ob * W + w
            planes[q]["z"] = float(zs[z_idx[ob]])
            planes[q]["wavelength"] = field.spectrum.wavelength[w]
            planes[q]["dy"], planes[q]["dx"] = field.dx_wv[w]
            planes[q]["shift_y"], planes[q]["shift_x"] = shift_yx
            planes[q]["in_plane"] = int(in_idx[ob]) * W + w
            planes[q]["h_plane"] = int(h_index[q]) if h_index is not None else 0
    return planes, out_batch, nb_in, nb_out


@pytest.mark.parametrize("batch,W,zshape,h", [((), 1, (), False), ((4,), 1, (), False), ((2, 3), 3, (), False),
                                              ((), 3, (5, 1, 1), False), ((2,), 1, (3, 1), True),
                                              ((3,), 2, (3,), True)])
def test_vectorised_plane_table_matches_plane_by_plane(batch, W, zshape, h):
    f = _stub(batch, W, [[0.3, 0.25]] if W == 1 else [[0.3 + 0.01 * w, 0.25] for w in range(W)],
              np.linspace(0.45, 0.63, W))
    zs = np.linspace(-5.0, 7.0, int(np.prod(zshape)) if zshape else 1)
    nb_out = int(np.prod(np.broadcast_shapes(tuple(batch), zshape))) if (batch or zshape) else 1
    h_index = (np.arange(nb_out * W)[::-1] % 4) if h else None
    got = P._plan_planes(f, zs, zshape, 256, 256, shift_yx=(1.5, -2.0), h_index=h_index)
    ref = _loop_planes(f, zs, zshape, (1.5, -2.0), h_index)
    assert got[1:] == ref[1:]
    assert got[0].tobytes() == ref[0].tobytes()
