"""Parity at the benchmark configurations' full sizes against the FP64 oracle.

* Differentiable multislice: 256 slices of 1024^2, dn Gaussian-filtered
  (sigma 4 px, periodic) N(0, 0.02), alpha ~ U[0, 0.05] (absorption =
  alpha / (k0 dz)), dz 0.2 um, spacing 0.1 um, lambda 0.532 um, n 1.33,
  plane-wave input, L2 loss against a seeded target, checkpoint every 16:
  forward relative L2 <= 1e-5, dL/d dn and the loss <= 1e-4.
* Modified Born series: 256^3 interior with 200 random spheres (radius
  U[0.5, 3] um, n U[1.36, 1.45]) in n = 1.33, 32-voxel absorbing boundary
  (320^3), spacing 0.1 um, lambda 0.5 um, y-polarised current sheet at
  x-index 34: one update from the preconditioned source and one from an
  arbitrary iterate, relative L2 <= 2e-5 (the per-update bar of the small
  grids).
* Serving: requests of every side {256, 512, 1024, 2048} and every op in one
  mixed stream, each result identical to the lone call; a sample of them
  against the FP64 oracle at 1e-5.

The oracle runs on all host cores (scipy.fft workers).
"""

import os

import numpy as np
import pytest

from oracle import chromatix_oracle as O
from tests.helpers import rel, to_np

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _workers():
    O.set_fft_workers(os.cpu_count())
    yield
    O.set_fft_workers(None)


def _gaussian_filtered(rng, shape, sigma, scale):
    x = rng.standard_normal(shape) * scale
    fy = np.fft.fftfreq(shape[-2])[:, None]
    fx = np.fft.fftfreq(shape[-1])[None, :]
    g = np.exp(-2 * (np.pi * sigma) ** 2 * (fy**2 + fx**2))
    import scipy.fft as sfft

    return np.real(sfft.ifft2(sfft.fft2(x, axes=(-2, -1), workers=os.cpu_count()) * g, axes=(-2, -1),
                              workers=os.cpu_count()))


def test_multislice_256_slices_1024_forward_and_gradient():
    import torch

    import chromatix_b200.functional as cf

    D, N, dz, lam, dx, n = 256, 1024, 0.2, 0.532, 0.1, 1.33
    rng = np.random.default_rng(0)
    dn = _gaussian_filtered(rng, (D, N, N), 4.0, 0.02).astype(np.float32)
    k0 = 2 * np.pi / lam
    ab = (rng.uniform(0, 0.05, (D, N, N)) / (k0 * dz)).astype(np.float32)
    pw = cf.plane_wave((N, N), dx, lam)
    u0 = to_np(pw.u)
    I0 = float(np.mean(np.abs(u0) ** 2))
    target = np.random.default_rng(1).uniform(0.5, 1.5, (N, N)) * I0
    L64, gdn64, _, uout64 = O.multislice_loss_and_grad(u0.astype(np.complex128), dn.astype(np.float64),
                                                       ab.astype(np.float64), target, n, dz, lam, dx)
    dn_t = torch.as_tensor(dn, device="cuda").requires_grad_(True)
    ab_t = torch.as_tensor(ab, device="cuda")
    out = cf.multislice_thick_sample(pw, ab_t, dn_t, n, dz, 0, checkpoint_every=16)
    e_fwd = rel(to_np(out.u), uout64)
    assert e_fwd < 1e-5, e_fwd
    loss = ((out.u.real ** 2 + out.u.imag ** 2 - torch.as_tensor(target, device="cuda", dtype=torch.float32)) ** 2)
    loss = loss.sum()
    loss.backward()
    assert abs(float(loss) - L64) / L64 < 1e-4
    e_g = rel(to_np(dn_t.grad), gdn64)
    assert e_g < 1e-4, e_g


def _c5_problem():
    """The 320^3 benchmark problem (host arrays, FP64)."""
    rng = np.random.default_rng(0)
    n_in, sp = 256, 0.1
    ax = (np.arange(n_in) - n_in // 2) * sp
    n = np.full((n_in,) * 3, 1.33)
    for _ in range(200):
        c = rng.uniform(ax[0], ax[-1], 3)
        r = rng.uniform(0.5, 3.0)
        ni = rng.uniform(1.36, 1.45)
        lo = [max(0, int(np.floor((c[d] - r - ax[0]) / sp))) for d in range(3)]
        hi = [min(n_in, int(np.ceil((c[d] + r - ax[0]) / sp)) + 1) for d in range(3)]
        sl = tuple(slice(lo[d], hi[d]) for d in range(3))
        gx, gy, gz = np.meshgrid(ax[sl[0]], ax[sl[1]], ax[sl[2]], indexing="ij")
        m = (gx - c[0]) ** 2 + (gy - c[1]) ** 2 + (gz - c[2]) ** 2 <= r * r
        n[sl][m] = ni
    perm, _ = O.mbs_add_absorbing_bc((n**2).astype(np.complex128), sp, (0, 1, 2), 3.2, 0.25, 1.33)
    J = np.zeros(perm.shape + (3,), np.complex128)
    J[34, :, :, 1] = 1.0
    k0 = 2 * np.pi / 0.5
    return perm, O.mbs_source_field(J, k0), sp, k0


def test_mbs_updates_at_320_cubed():
    import torch

    from chromatix_b200.experimental import mbs

    perm, src, sp, k0 = _c5_problem()
    assert perm.shape == (320, 320, 320)
    op = O.MBSOperator(perm, sp, k0, src)
    sample = mbs.Sample(torch.as_tensor(perm.astype(np.complex64), device="cuda"), sp)
    source = mbs.Source(torch.zeros(perm.shape + (3,), dtype=torch.complex64, device="cuda"), k0)
    source.field = torch.as_tensor(src.astype(np.complex64), device="cuda")
    E1, info = mbs.solve(sample, source, shift=op.bias, scale=op.scale, maxiter=1, tol=0.0, return_info=True)
    assert abs(info["num_scale"] - op.num_scale) / op.num_scale < 1e-5
    ref1 = op.step(op.prec_y) * op.num_scale
    e1 = rel(to_np(E1), ref1)
    assert e1 < 2e-5, e1
    del E1, ref1
    x0 = (np.random.default_rng(3).standard_normal(perm.shape + (3,)).astype(np.float32)
          + 1j * np.random.default_rng(4).standard_normal(perm.shape + (3,)).astype(np.float32))
    x0 = (x0 * np.float32(op.num_scale)).astype(np.complex64)
    E2, _ = mbs.solve(sample, source, shift=op.bias, scale=op.scale, maxiter=1, tol=0.0, return_info=True,
                      initial_E=torch.as_tensor(x0, device="cuda"))
    ref2 = op.step(x0.astype(np.complex128) / op.num_scale) * op.num_scale
    e2 = rel(to_np(E2), ref2)
    assert e2 < 2e-5, e2


def test_serving_mix_of_every_side_matches_lone_calls_and_oracle():
    import torch

    import chromatix_b200.functional as cf
    from chromatix_b200.core.field import Field
    from chromatix_b200.serving import PropagationServer, Request

    rng = np.random.default_rng(0)
    sides = (256, 512, 1024, 2048)
    fields = {}
    for n in sides:
        ph = rng.uniform(0, 2 * np.pi, (n, n))
        fields[n] = torch.as_tensor(np.exp(1j * ph).astype(np.complex64), device="cuda")
    srv = PropagationServer(budget_bytes=60e9, n_streams=4, max_batch=8)
    reqs = []
    for i in range(36):
        n = sides[i % 4]
        op = ("asm", "transfer", "czt_zoom")[(i // 4) % 3]
        r = Request(op=op, u=fields[n], dx=0.3, z=float(rng.uniform(1, 500)), wavelength=float(rng.uniform(0.4, 0.7)),
                    zoom=float(rng.uniform(0.25, 4)), out_shape=(512, 512))
        reqs.append(srv.submit(r))
        if i % 5 == 0:
            srv.step()
    srv.drain()
    torch.cuda.synchronize()

    def alone(r):
        f = Field.build(r.u, r.dx, r.wavelength)
        N = r.side
        if r.op == "asm":
            return cf.asm_propagate(f, r.z, r.n, N // 2, mode="same").u
        if r.op == "transfer":
            return cf.transfer_propagate(f, r.z, r.n, N // 2, mode="same").u
        return cf.asm_propagate(f, r.z, r.n, N // 2, output_dx=np.array([r.dx / r.zoom] * 2),
                                output_shape=r.out_shape).u

    for r in reqs:
        ref = alone(r)
        torch.cuda.synchronize()
        assert torch.equal(r.out, ref), (r.op, r.side)
    checked = 0
    for r in reqs:
        if r.side > 1024 or checked >= 6:
            continue
        u = to_np(r.u)
        f = O.field_build(u, r.dx, r.wavelength)
        N = r.side
        if r.op == "asm":
            ref = O.asm_propagate(f, r.z, r.n, N // 2, mode="same").u
            tol = 1e-5
        elif r.op == "transfer":
            ref = O.transfer_propagate(f, r.z, r.n, N // 2, mode="same").u
            tol = 1e-5
        else:
            ref = O.asm_propagate(f, r.z, r.n, N // 2, output_dx=np.array([r.dx / r.zoom] * 2),
                                  output_shape=r.out_shape).u
            tol = 1e-5
        e = rel(to_np(r.out), ref)
        assert e < tol, (r.op, r.side, e)
        checked += 1
