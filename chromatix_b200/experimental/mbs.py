"""Modified Born series (experimental/modified_born_series/).

``Sample``, ``EmptySample``, ``Source``, ``add_absorbing_bc``,
``get_shift_and_scale`` and ``solve`` keep the reference's names and argument
meanings.  The fixed-point iteration runs in fused CUDA passes
(``cx_mbs_iterate``): three component planes of the field stay resident in
HBM, the 3D FFTs are split into z / y / x passes with the preconditioner's
scattering potential and Green's-function division fused in, and the
convergence test reads FP64 residual sums accumulated on the device.
``use_bicgstab=True`` runs BiCGStab on the same operator (``cx_mbs_forward``)
with native FP64-accumulated inner products and fused vector updates.
"""

from __future__ import annotations

import math

import numpy as np
from scipy import constants as _const

from .. import _native as nat

__all__ = ["Sample", "EmptySample", "Source", "add_absorbing_bc", "get_shift_and_scale", "solve"]


class cx_mbs_desc(nat.ctypes.Structure):
    _fields_ = [("X", nat.c_int32), ("Y", nat.c_int32), ("Z", nat.c_int32), ("spacing", nat.c_double),
                ("k0", nat.c_double), ("s_re", nat.c_double), ("s_im", nat.c_double), ("kb2_re", nat.c_double),
                ("kb2_im", nat.c_double)]


_SIG = False


def _lib():
    global _SIG
    L = nat.lib()
    if not _SIG:
        P = nat.ctypes.POINTER(cx_mbs_desc)
        V = nat.c_void_p
        L.cx_mbs_workspace_size.restype = nat.c_int32
        L.cx_mbs_workspace_size.argtypes = [P, nat.ctypes.POINTER(nat.c_size_t)]
        L.cx_mbs_precondition.restype = nat.c_int32
        L.cx_mbs_precondition.argtypes = [P, V, V, V, V, nat.c_size_t, V]
        L.cx_mbs_iterate.restype = nat.c_int32
        L.cx_mbs_iterate.argtypes = [P, V, V, V, V, V, V, nat.c_size_t, V]
        L.cx_mbs_forward.restype = nat.c_int32
        L.cx_mbs_forward.argtypes = [P, V, V, V, V, nat.c_size_t, V]
        L.cx_cvec_dot.restype = nat.c_int32
        L.cx_cvec_dot.argtypes = [V, V, nat.ctypes.c_int64, V, V]
        L.cx_cvec_lincomb.restype = nat.c_int32
        L.cx_cvec_lincomb.argtypes = [nat.ctypes.c_int64, nat.ctypes.POINTER(nat.c_double), V, V, V, V, V, V]
        _SIG = True
    return L


class Sample:
    """Permittivity on a uniform grid (experimental/modified_born_series/sample.py:9-68)."""

    def __init__(self, permittivity, spacing: float):
        torch = nat.torch_mod()
        if not isinstance(permittivity, torch.Tensor):
            permittivity = torch.as_tensor(np.asarray(permittivity), device="cuda")
        self.permittivity = permittivity
        self.spacing = float(spacing)
        self.ROI = tuple(slice(0, s) for s in self.shape)

    @property
    def shape(self):
        return tuple(self.permittivity.shape)

    @property
    def grid(self):
        torch = nat.torch_mod()
        axes = [np.arange(N) - (N // 2 if N != 1 else 0) for N in self.shape]
        g = np.stack(np.meshgrid(*axes, indexing="ij"), axis=-1) * self.spacing
        return torch.as_tensor(g.astype(np.float32), device=self.permittivity.device)

    @property
    def k_grid(self):
        torch = nat.torch_mod()
        g = np.stack(np.meshgrid(*[np.fft.fftfreq(N) for N in self.shape], indexing="ij"), axis=-1)
        return torch.as_tensor((2 * np.pi * g / self.spacing).astype(np.float32), device=self.permittivity.device)

    @property
    def extent(self):
        return np.asarray(self.shape) * self.spacing

    def replace(self, **kw) -> "Sample":
        new = Sample.__new__(Sample)
        new.__dict__.update(self.__dict__)
        new.__dict__.update(kw)
        return new


def EmptySample(shape, spacing: float) -> Sample:
    torch = nat.torch_mod()
    return Sample(torch.zeros(tuple(shape), dtype=torch.complex64, device="cuda"), spacing)


class Source:
    """``field = -1j / k0 * 1e-6 * c * mu_0 * J`` (sample.py:75-85)."""

    def __init__(self, current_density, k0: float):
        torch = nat.torch_mod()
        if not isinstance(current_density, torch.Tensor):
            current_density = torch.as_tensor(np.asarray(current_density), device="cuda")
        self.k0 = float(k0)
        self.field = (current_density.to(torch.complex64) * complex(-1j / self.k0 * 1e-6 * _const.c * _const.mu_0))

    @property
    def current_density(self):
        return self.field / complex(-1j / self.k0 * 1e-6 * _const.c * _const.mu_0)


def add_absorbing_bc(sample: Sample, axis, thickness: float, max_extinction: float = 0.25,
                     n_background: float = 1.0) -> Sample:
    """Linear-ramp extinction boundary (sample.py:88-124)."""
    torch = nat.torch_mod()
    if not isinstance(axis, tuple):
        axis = (axis,)
    bw = int(thickness / sample.spacing)
    bs = tuple((bw, bw) if i in axis else (0, 0) for i in range(3))
    ext = np.pad(np.zeros(sample.shape), bs, mode="linear_ramp", end_values=max_extinction)
    eps_b = (n_background + 1j * ext) ** 2 - n_background**2
    perm = torch.nn.functional.pad(
        torch.view_as_real(sample.permittivity.to(torch.complex64)).movedim(-1, 0),
        tuple(v for pair in reversed(bs) for v in pair), value=0.0).movedim(0, -1)
    perm = torch.view_as_complex(perm.contiguous())
    # constant padding with n_background^2 (real part)
    mask = np.pad(np.zeros(sample.shape, dtype=bool), bs, constant_values=True)
    perm = perm + torch.as_tensor(np.where(mask, n_background**2, 0.0).astype(np.complex64), device=perm.device)
    perm = perm + torch.as_tensor(eps_b.astype(np.complex64), device=perm.device)
    roi = tuple(slice(w, w + s) for (w, _), s in zip(bs, sample.shape))
    out = sample.replace(permittivity=perm)
    out.ROI = roi
    return out


def _min_enclosing_circle(pts):
    pts = [complex(p) for p in pts]
    rng = np.random.default_rng(0)
    rng.shuffle(pts)

    def c2(a, b):
        c = (a + b) / 2
        return c, abs(a - c)

    def c3(a, b, c):
        ax, ay, bx, by, cx, cy = a.real, a.imag, b.real, b.imag, c.real, c.imag
        d = 2 * (ax * (by - cy) + bx * (cy - ay) + cx * (ay - by))
        if abs(d) < 1e-300:
            return max((c2(a, b), c2(a, c), c2(b, c)), key=lambda t: t[1])
        ux = ((ax**2 + ay**2) * (by - cy) + (bx**2 + by**2) * (cy - ay) + (cx**2 + cy**2) * (ay - by)) / d
        uy = ((ax**2 + ay**2) * (cx - bx) + (bx**2 + by**2) * (ax - cx) + (cx**2 + cy**2) * (bx - ax)) / d
        ctr = complex(ux, uy)
        return ctr, abs(a - ctr)

    def inside(cr, p):
        return abs(p - cr[0]) <= cr[1] * (1 + 1e-12) + 1e-15

    cr = (pts[0], 0.0)
    for i in range(1, len(pts)):
        if inside(cr, pts[i]):
            continue
        cr = (pts[i], 0.0)
        for j in range(i):
            if inside(cr, pts[j]):
                continue
            cr = c2(pts[i], pts[j])
            for k in range(j):
                if not inside(cr, pts[k]):
                    cr = c3(pts[i], pts[j], pts[k])
    return cr


def get_shift_and_scale(permittivity, n_directions: int = 64):
    """Shift and scale of the preconditioner (solver.py:10-39).

    The reference minimises ``max|eps - s|^2`` with optimistix NonlinearCG;
    here the centre of the smallest circle enclosing the ``n_directions``
    extreme points of the permittivity values (a near-optimal shift) is used,
    and the scale is ``1.1i`` times the exact maximum distance from it, which
    keeps the iteration's convergence guarantee.  Returns ``(shift, 1/scale)``.
    """
    torch = nat.torch_mod()
    e = permittivity.reshape(-1).to(torch.complex64)
    er, ei = e.real, e.imag
    pts = []
    for k in range(n_directions):
        t = 2 * math.pi * k / n_directions
        proj = er * math.cos(t) + ei * math.sin(t)
        pts.append(complex(e[int(torch.argmax(proj))].item()))
    c, _ = _min_enclosing_circle(np.unique(np.asarray(pts)))
    R = float(torch.max((e - complex(c)).abs()).item())
    scale = 1.1j * R
    return complex(c), 1.0 / scale


def _planes(v):
    """(X, Y, Z, 3) -> contiguous (3, X, Y, Z)."""
    return v.movedim(-1, 0).contiguous()


def solve(sample: Sample, source: Source, initial_E=None, maxiter: int = 1000, tol: float = 1e-3,
          implicit_diff: bool = True, use_bicgstab: bool = False, *, rtol: float | None = None,
          shift=None, scale=None, return_info: bool = False):
    """Electric field of the scattering problem (solver.py:101-146).

    ``use_bicgstab=True``: BiCGStab on ``prec_forward(x) = prec_y``
    (solver.py:143-144), stopping at ||r|| <= tol ||prec_y|| (``rtol`` in
    place of tol when given) -- see ``_bicgstab``.  Otherwise the
    fixed-point iteration ``x <- prec_y - prec_forward(x) + x``.  Stops when
    ``||x_{k+1} - x_k||_2 <= tol`` (the absolute rule of jaxopt's
    FixedPointIteration, which the reference uses) or, if ``rtol`` is given,
    when ``||x_{k+1} - x_k|| / ||x_{k+1}|| < rtol``; both norms are FP64 sums
    accumulated on the device.  Returns E of shape (X, Y, Z, 3).
    """
    torch = nat.torch_mod()
    nat.refuse_grad("modified Born series solve", sample.permittivity, source.field)
    eps = sample.permittivity.to(torch.complex64).contiguous()
    nat.require_cuda(eps, "permittivity")
    X, Y, Z = eps.shape
    if shift is None or scale is None:
        shift, scale = get_shift_and_scale(eps)
    kb2 = complex(shift) * complex(scale) + 1.0
    d = cx_mbs_desc()
    d.X, d.Y, d.Z = X, Y, Z
    d.spacing, d.k0 = sample.spacing, source.k0
    d.s_re, d.s_im = complex(scale).real, complex(scale).imag
    d.kb2_re, d.kb2_im = kb2.real, kb2.imag
    L = _lib()
    ws_b = nat.c_size_t(0)
    nat.check(L.cx_mbs_workspace_size(d, ws_b))
    dev = eps.device
    ws = nat.workspace(ws_b.value, dev)
    st = nat.stream_handle(dev)
    src = _planes(source.field.to(torch.complex64).to(dev))
    prec_y = torch.empty_like(src)
    nat.check(L.cx_mbs_precondition(d, nat.ptr(eps), nat.ptr(src), nat.ptr(prec_y), nat.ptr(ws), ws_b.value, st))
    num_scale = float(prec_y.abs().max().item())
    prec_y /= num_scale
    x = prec_y.clone() if initial_E is None else _planes(initial_E.to(torch.complex64)) / num_scale
    if use_bicgstab:
        x, info = _bicgstab(L, d, eps, prec_y, x, ws, ws_b.value, st, maxiter, tol, rtol)
        E = (x * num_scale).movedim(0, -1).contiguous()
        if return_info:
            info.update({"shift": shift, "scale": scale, "num_scale": num_scale})
            return E, info
        return E
    x_new = torch.empty_like(x)
    acc = torch.zeros(2, dtype=torch.float64, device=dev)
    acc_h = torch.zeros(2, dtype=torch.float64).pin_memory()
    done = torch.cuda.Event()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    it, res_abs, res_rel = 0, float("inf"), float("inf")
    for it in range(1, maxiter + 1):
        nat.check(L.cx_mbs_iterate(d, nat.ptr(eps), nat.ptr(prec_y), nat.ptr(x), nat.ptr(x_new), nat.ptr(acc),
                                   nat.ptr(ws), ws_b.value, st))
        x, x_new = x_new, x
        acc_h.copy_(acc, non_blocking=True)
        done.record()
        done.synchronize()
        a = acc_h.numpy()
        res_abs = math.sqrt(a[0])
        res_rel = math.sqrt(a[0] / a[1]) if a[1] > 0 else float("inf")
        if res_abs <= tol or (rtol is not None and res_rel < rtol):
            break
    ev1.record()
    E = (x * num_scale).movedim(0, -1).contiguous()
    if return_info:
        ev1.synchronize()
        return E, {"iterations": it, "residual_abs": res_abs, "residual_rel": res_rel, "shift": shift,
                   "scale": scale, "num_scale": num_scale, "loop_ms": ev0.elapsed_time(ev1)}
    return E


class _Krylov:
    """Native complex vector algebra on the device (FP64 inner products read
    back through page-locked memory)."""

    def __init__(self, L, n, dev, st):
        torch = nat.torch_mod()
        self.L, self.n, self.st = L, int(n), st
        self.acc = torch.zeros(4, dtype=torch.float64, device=dev)
        self.nrm = torch.zeros(1, dtype=torch.float64, device=dev)
        self.host = torch.zeros(4, dtype=torch.float64).pin_memory()
        self.ev = torch.cuda.Event()

    def _read(self, t, k):
        self.host[:k].copy_(t[:k], non_blocking=True)
        self.ev.record()
        self.ev.synchronize()
        return self.host[:k].numpy().copy()

    def dot(self, x, y):
        """(sum conj(x) y, sum |x|^2, sum |y|^2) in FP64."""
        nat.check(self.L.cx_cvec_dot(nat.ptr(x), nat.ptr(y), self.n, nat.ptr(self.acc), self.st))
        a = self._read(self.acc, 4)
        return complex(a[0], a[1]), float(a[2]), float(a[3])

    def comb(self, out, c0, x, c1, y, c2=0.0, z=None, norm=False):
        """out = c0 x + c1 y [+ c2 z]; returns sum |out|^2 when ``norm``."""
        c = (nat.c_double * 6)(complex(c0).real, complex(c0).imag, complex(c1).real, complex(c1).imag,
                               complex(c2).real, complex(c2).imag)
        nat.check(self.L.cx_cvec_lincomb(self.n, c, nat.ptr(x), nat.ptr(y), nat.ptr(z), nat.ptr(out),
                                         nat.ptr(self.nrm) if norm else None, self.st))
        return float(self._read(self.nrm, 1)[0]) if norm else None


def _bicgstab(L, d, eps, b, x, ws, ws_bytes, st, maxiter, tol, rtol):
    """BiCGStab on prec_forward(x) = prec_y (solver.py:143-144).

    The reference calls jax.scipy.sparse.linalg.bicgstab (unpreconditioned:
    the series' preconditioning is already in prec_forward); this is the same
    published algorithm (van der Vorst, SIAM J. Sci. Stat. Comput. 13, 1992),
    with its stopping rule ||r|| <= max(tol ||b||, 0) (``rtol`` overrides
    tol when given) and its breakdown exits (rho = 0, alpha = 0 or
    omega = 0 end the loop).  Matrix-vector products are ``cx_mbs_forward``;
    inner products accumulate in FP64 on the device."""
    torch = nat.torch_mod()
    n = x.numel()
    K = _Krylov(L, n, x.device, st)

    def A(v, out):
        nat.check(L.cx_mbs_forward(d, nat.ptr(eps), nat.ptr(v), nat.ptr(out), nat.ptr(ws), ws_bytes, st))

    q = torch.empty_like(x)
    A(x, q)
    r = torch.empty_like(x)
    rs = K.comb(r, 1.0, b, -1.0, q, norm=True)
    _, bs, _ = K.dot(b, b)
    thr2 = (rtol if rtol is not None else tol) ** 2 * bs
    rhat = r.clone()
    p, q = r.clone(), r.clone()
    s_, t = torch.empty_like(x), torch.empty_like(x)
    rho = alpha = omega = 1.0 + 0j
    it, status = 0, "maxiter"
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    while rs > thr2 and it < maxiter:
        rho_new, _, _ = K.dot(rhat, r)
        if rho_new == 0:
            status = "breakdown (rho = 0)"
            break
        beta = rho_new / rho * alpha / omega
        K.comb(p, 1.0, r, beta, p, -beta * omega, q)  # p = r + beta (p - omega q)
        A(p, q)
        rq, _, _ = K.dot(rhat, q)
        alpha = rho_new / rq
        ss = K.comb(s_, 1.0, r, -alpha, q, norm=True)  # s = r - alpha q
        it += 1
        if ss < thr2:  # early exit: x + alpha p already meets the tolerance
            K.comb(x, 1.0, x, alpha, p)
            r, s_ = s_, r
            rs = ss
            break
        A(s_, t)
        ts, tt, _ = K.dot(t, s_)
        omega = ts / tt
        K.comb(x, 1.0, x, alpha, p, omega, s_)  # x += alpha p + omega s
        rs = K.comb(r, 1.0, s_, -omega, t, norm=True)  # r = s - omega t
        rho = rho_new
        if alpha == 0 or omega == 0:
            status = "breakdown (alpha or omega = 0)"
            break
    else:
        status = "converged" if rs <= thr2 else "maxiter"
    if rs <= thr2:
        status = "converged"
    ev1.record()
    ev1.synchronize()
    res_rel = math.sqrt(rs / bs) if bs > 0 else float("inf")
    return x, {"iterations": it, "residual_abs": math.sqrt(rs), "residual_rel": res_rel, "status": status,
               "solver": "bicgstab", "loop_ms": ev0.elapsed_time(ev1)}
