"""The oracle's birefringent multislice (functional/samples.py:444-546): the
reference has no test of it, so the restatement is pinned by exact
properties -- one slice is affine in the potential (u(V) = P u + H V Q u),
the projector Q is transverse (k . (Q x) = 0 for propagating k), a zero
potential with NA 0 passes only the DC term -- and by a second, literal
restatement with explicit DFT matrices and per-frequency loops (no GPU)."""

import numpy as np

from oracle import chromatix_oracle as O


def _u(shape, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(shape + (3,)) + 1j * rng.standard_normal(shape + (3,))


def test_one_slice_is_affine_in_the_potential():
    u = _u((12, 10), 0)
    V = np.random.default_rng(1).uniform(-0.05, 0.05, (1, 12, 10, 3, 3))
    a = O.polarized_multislice_thick_sample(u, 0.3, 0.532, 0 * V, 1.33, 0.5)
    b = O.polarized_multislice_thick_sample(u, 0.3, 0.532, V, 1.33, 0.5)
    c = O.polarized_multislice_thick_sample(u, 0.3, 0.532, 2.5 * V, 1.33, 0.5)
    assert O.rel_l2(c - a, 2.5 * (b - a)) < 1e-12
    assert O.rel_l2(b, a) > 1e-4


def test_zero_na_blocks_the_field():
    u = _u((8, 8), 2)
    out = O.polarized_multislice_thick_sample(u, 0.3, 0.532, np.zeros((2, 8, 8, 3, 3)), 1.0, 0.5, NA=0.0)
    # only the DC column passes an NA of 0 (|k_perp| = 0 <= 0): a constant field
    np.testing.assert_allclose(out, np.broadcast_to(out[:1, :1], out.shape), atol=1e-12)


def test_projector_is_transverse():
    km = 2 * np.pi * 1.33 / 0.532
    rng = np.random.default_rng(3)
    for _ in range(20):
        kp = rng.uniform(-0.9, 0.9, 2) * km / np.sqrt(2)
        k = np.array([np.sqrt(km**2 - kp @ kp), *kp]) / km
        Q = np.eye(3) - np.outer(k, k)
        x = rng.standard_normal(3) + 1j * rng.standard_normal(3)
        assert abs(k @ (Q @ x)) < 1e-12


def _independent_polarized(u, dx, lam, V, n, dz, NA):
    """The reference's slice step written out literally with explicit DFT
    matrices and per-frequency loops (no np.fft, no broadcasting tricks):
    Q_op, P_op, H_op as in functional/samples.py:477-512, padding to twice
    the size after the data, crop of the first rows and columns."""
    ny, nx = u.shape[:2]
    P, Qn = 2 * ny, 2 * nx
    Fy = np.exp(-2j * np.pi * np.outer(np.arange(P), np.arange(P)) / P)
    Fx = np.exp(-2j * np.pi * np.outer(np.arange(Qn), np.arange(Qn)) / Qn)

    def fft2(a):  # per component
        return np.stack([Fy @ a[..., c] @ Fx.T for c in range(3)], -1)

    def ifft2(a):
        return np.stack([Fy.conj() @ a[..., c] @ Fx.conj().T / (P * Qn) for c in range(3)], -1)

    def freq(j, N, d):  # fftfreq(N, d)[j], N even
        return (j if j < N // 2 else j - N) / (N * d)

    km = 2 * np.pi * n / lam
    Qm = np.zeros((P, Qn, 3, 3))
    e = np.zeros((P, Qn), complex)
    h = np.zeros((P, Qn), complex)
    for a in range(P):
        for b in range(Qn):
            ky, kx = 2 * np.pi * freq(a, P, dx), 2 * np.pi * freq(b, Qn, dx)
            kz = np.sqrt(max(0.0, km**2 - ky**2 - kx**2))
            if ky**2 + kx**2 <= NA**2 * km**2:
                k = np.array([kz, ky, kx]) / km
                Qm[a, b] = np.eye(3) - np.outer(k, k)
            if kz > 0:
                e[a, b] = np.exp(1j * kz * dz)
                h[a, b] = -1j / 2 * np.exp(1j * kz * dz) / kz * dz

    def pad(a):
        out = np.zeros((P, Qn, 3), complex)
        out[:ny, :nx] = a
        return out

    def apply(M, a):
        return np.einsum("abij,abj->abi", M, a)

    for Vi in V:
        q_u = ifft2(apply(Qm, fft2(pad(u))))[:ny, :nx]
        s = np.einsum("abij,abj->abi", Vi, q_u)
        p_u = ifft2(apply(Qm, e[..., None] * fft2(pad(u))))[:ny, :nx]
        h_s = ifft2(apply(Qm, h[..., None] * fft2(pad(s))))[:ny, :nx]
        u = p_u + h_s
    return u


def test_restatement_matches_an_independent_one():
    rng = np.random.default_rng(5)
    for (ny, nx), NA, lam in [((4, 6), 1.0, 0.55), ((6, 4), 0.7, 0.6)]:
        u = _u((ny, nx), 6)
        V = rng.uniform(-0.1, 0.1, (2, ny, nx, 3, 3))
        a = O.polarized_multislice_thick_sample(u, 0.2, lam, V, 1.33, 0.4, NA)
        b = _independent_polarized(u, 0.2, lam, V, 1.33, 0.4, NA)
        assert O.rel_l2(a, b) < 1e-12
