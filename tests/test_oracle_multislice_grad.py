"""The FP64 multislice adjoint of the oracle vs central finite differences
(pins the gradient the CUDA adjoint is checked against)."""

import numpy as np

from oracle import chromatix_oracle as O


def test_oracle_adjoint_central_differences():
    rng = np.random.default_rng(0)
    ny, nx, D = 16, 24, 5
    lam, dz, n, dx = 0.532, 0.2, 1.33, 0.1
    u = (rng.uniform(0.9, 1, (ny, nx)) * np.exp(1j * rng.uniform(0, 2 * np.pi, (ny, nx))))
    dn = 0.02 * rng.standard_normal((D, ny, nx))
    ab = rng.uniform(0, 0.05, (D, ny, nx))
    target = rng.uniform(0.5, 1.5, (ny, nx))
    L, gdn, gab, _ = O.multislice_loss_and_grad(u, dn, ab, target, n, dz, lam, dx, NA=0.9)
    h = 1e-6
    for _ in range(8):
        i, y, x = rng.integers(D), rng.integers(ny), rng.integers(nx)
        for arr, g in ((dn, gdn), (ab, gab)):
            p = arr.copy()
            m = arr.copy()
            p[i, y, x] += h
            m[i, y, x] -= h
            args = (p, ab) if arr is dn else (dn, p)
            argm = (m, ab) if arr is dn else (dn, m)
            Lp = O.multislice_loss_and_grad(u, *args, target, n, dz, lam, dx, NA=0.9)[0]
            Lm = O.multislice_loss_and_grad(u, *argm, target, n, dz, lam, dx, NA=0.9)[0]
            fd = (Lp - Lm) / (2 * h)
            assert abs(g[i, y, x] - fd) < 1e-6 * max(1.0, abs(fd)), (g[i, y, x], fd)


def test_oracle_loss_matches_forward():
    rng = np.random.default_rng(1)
    ny, nx, D = 16, 16, 3
    u = np.exp(1j * rng.uniform(0, 2 * np.pi, (ny, nx)))
    dn = 0.01 * rng.standard_normal((D, ny, nx))
    ab = np.zeros((D, ny, nx))
    f = O.field_build(u, 0.1, 0.532)
    out = O.multislice_thick_sample(f, ab, dn, 1.33, 0.2, 0)
    _, _, _, u_out = O.multislice_loss_and_grad(u, dn, ab, np.zeros((ny, nx)), 1.33, 0.2, 0.532, 0.1)
    assert O.rel_l2(u_out, out.u) < 1e-12
