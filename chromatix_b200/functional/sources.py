"""Sources (functional/sources.py) with lazy fusion into the PSF kernel.

``objective_point_source`` returns a lazily evaluated field.  ``phase_change``
and a forward ``ff_lens`` applied to it stay lazy, and reading ``.intensity``
of the result runs the fused batched-PSF pipeline (``cx_psf_4f``): the
source, pupil, power normalisation, phase mask and lens normalisation are
evaluated inside the FFT loader and only the intensity is written to HBM.
Reading ``.u`` (or applying any other operation) materialises the field with
the same kernels (``cx_psf_source`` then ``cx_optical_fft``).
"""

from __future__ import annotations

import numpy as np

from .. import _native as nat
from .. import config
from ..core.field import ChromaticScalarField, Field, ScalarField, _broadcast_dx
from ..core.spectrum import MonoSpectrum, Spectrum

__all__ = ["objective_point_source", "plane_wave", "materialize", "LazySourceField"]

_SIG = False


def _sigs(L):
    global _SIG
    if not _SIG:
        for name in ("cx_psf_source",):
            fn = getattr(L, name)
            fn.restype = nat.c_int32
            fn.argtypes = [nat.ctypes.POINTER(nat.cx_psf_desc), nat.ctypes.POINTER(nat.cx_psf_spectrum),
                           nat.c_void_p, nat.c_void_p, nat.c_void_p, nat.c_void_p, nat.c_size_t, nat.c_void_p]
        P, S = nat.ctypes.POINTER(nat.cx_psf_desc), nat.ctypes.POINTER(nat.cx_psf_spectrum)
        L.cx_psf_host_workspace_size.restype = nat.c_int32
        L.cx_psf_host_workspace_size.argtypes = [P, S, nat.ctypes.POINTER(nat.c_size_t)]
        L.cx_psf_4f_to_host.restype = nat.c_int32
        L.cx_psf_4f_to_host.argtypes = [P, S, nat.c_void_p, nat.c_void_p, nat.c_void_p, nat.c_void_p, nat.c_size_t,
                                        nat.c_void_p, nat.c_void_p]
        _SIG = True
    return L


class LazySourceField(Field):
    """A defocused point source behind an objective, not yet evaluated.

    Stages: ``"source"`` -> (``phase_change``) ``"phase"`` -> (``ff_lens``)
    ``"lens"``.  Layout and metadata are those of the equivalent eager field.
    """

    def __init__(self, recipe: dict, dx, spectrum: Spectrum, chromatic: bool, device):
        self._recipe = recipe
        self._u = None
        self.chromatic = chromatic
        self.spectrum = spectrum
        self.dx = dx
        self.origin = np.zeros((spectrum.size, 2)) if chromatic else np.zeros(2)
        self._device = device

    # -- metadata without evaluation ----------------------------------------
    @property
    def shape(self):
        r = self._recipe
        zb = (r["nz"],) if r["zbatch"] else ()
        return zb + tuple(r["shape"]) + ((self.spectrum.size,) if self.chromatic else ())

    @property
    def device(self):
        return self._device

    @property
    def stage(self) -> str:
        return self._recipe["stage"]

    @property
    def u(self):
        if self._u is None:
            self._u = self.materialized().u
        return self._u

    def replace(self, **kw) -> Field:
        return self.materialized().replace(**kw)

    # -- lazy composition ------------------------------------------------------
    def with_phase(self, phase, spectrally_modulate: bool) -> "LazySourceField":
        torch = nat.torch_mod()
        r = dict(self._recipe)
        ph = phase if isinstance(phase, torch.Tensor) else torch.as_tensor(np.asarray(phase))
        ph = ph.to(device=self._device, dtype=torch.float32).reshape(tuple(r["shape"])).contiguous()
        r["phase"] = ph
        r["spectrally_modulate"] = bool(spectrally_modulate)
        r["stage"] = "phase"
        return LazySourceField(r, self.dx, self.spectrum, self.chromatic, self._device)

    def with_lens(self, f: float, n: float, NA) -> "LazySourceField":
        r = dict(self._recipe)
        r["lens"] = (f, n, NA)
        r["stage"] = "lens"
        ny, nx = r["shape"]
        dxw = _broadcast_dx(self.dx, self.spectrum.size)
        L_sq = self.spectrum.wavelength * f / n
        du = np.stack([1.0 / (ny * dxw[:, 0]), 1.0 / (nx * dxw[:, 1])], axis=-1) * np.abs(L_sq)[:, None]
        dx = du if self.chromatic else du.reshape(2)
        return LazySourceField(r, dx, self.spectrum, self.chromatic, self._device)

    # -- evaluation ---------------------------------------------------------------
    def _desc(self):
        r = self._recipe
        d = nat.cx_psf_desc()
        ny, nx = r["shape"]
        d.ny, d.nx = ny, nx
        d.n_z = int(r["nz"])
        d.n_wv = self.spectrum.size
        # the fused pipeline's column pass has a tensor-core form at 1024 / 1280 rows
        tc = r.get("lens") is not None and ny in (1024, 1280) and nx % 8 == 0
        d.precision = config.precision_code(r["precision"], tensor_core=tc)
        d.has_phase = 1 if r.get("phase") is not None else 0
        d.spectrally_modulate = 1 if r.get("spectrally_modulate", True) else 0
        d.normalize_power = 0 if r["power"] is None else 1
        d.f_obj, d.n_medium, d.NA = r["f"], r["n"], r["NA"]
        d.power = 0.0 if r["power"] is None else float(r["power"])
        d.amplitude = float(r["amplitude"])
        d.offset_y, d.offset_x = r["offset"]
        lens = r.get("lens")
        if lens is not None:
            d.f_lens = lens[0]
            d.lens_NA = -1.0 if lens[2] is None else float(lens[2])
        else:
            d.f_lens = 1.0
            d.lens_NA = -1.0
        return d

    def _spec(self):
        r = self._recipe
        wl = np.ascontiguousarray(self.spectrum.wavelength, dtype=np.float64)
        dens = np.ascontiguousarray(self.spectrum.density if self.chromatic else np.ones(1), dtype=np.float64)
        dxw = _broadcast_dx(r["src_dx"], self.spectrum.size)
        dy = np.ascontiguousarray(dxw[:, 0])
        dx = np.ascontiguousarray(dxw[:, 1])
        keep = (wl, dens, dy, dx)
        P = nat.ctypes.POINTER(nat.c_double)
        s = nat.cx_psf_spectrum(wl.ctypes.data_as(P), dens.ctypes.data_as(P), dy.ctypes.data_as(P),
                                dx.ctypes.data_as(P))
        return s, keep

    def _z_dev(self):
        torch = nat.torch_mod()
        r = self._recipe
        if r.get("z_dev") is not None:
            return r["z_dev"]
        return nat.upload(np.ascontiguousarray(r["z"], dtype=np.float64), self._device)

    def _source_field(self) -> Field:
        """Materialise the source (+ phase) stage."""
        torch = nat.torch_mod()
        L = _sigs(nat.lib())
        r = self._recipe
        d = self._desc()
        spec, keep = self._spec()
        ny, nx = r["shape"]
        W = self.spectrum.size
        u = torch.empty((int(r["nz"]), ny, nx, W), dtype=torch.complex64, device=self._device)
        ws = nat.workspace(256, self._device)
        zd = self._z_dev()
        ph = r.get("phase")
        nat.check(L.cx_psf_source(d, spec, nat.ptr(zd), nat.ptr(ph), nat.ptr(u), nat.ptr(ws), 256,
                                  nat.stream_handle(self._device)))
        del keep
        if not r["zbatch"]:
            u = u[0]
        if not self.chromatic:
            u = u[..., 0]
        src_dx = _broadcast_dx(r["src_dx"], W)
        if self.chromatic:
            return ChromaticScalarField(u.contiguous(), src_dx, 0.0, self.spectrum)
        return ScalarField(u.contiguous(), src_dx.reshape(2), 0.0, self.spectrum)

    def materialized(self) -> Field:
        src = self._source_field()
        lens = self._recipe.get("lens")
        if lens is None:
            return src
        from .lenses import ff_lens

        return ff_lens(src, lens[0], lens[1], lens[2], precision=self._recipe["precision"])

    @property
    def intensity(self):
        if self.stage != "lens" or self._u is not None:
            return super().intensity
        torch = nat.torch_mod()
        r = self._recipe
        L = nat.lib()
        d = self._desc()
        spec, keep = self._spec()
        ws_b = nat.c_size_t(0)
        nat.check(L.cx_psf_workspace_size(d, ws_b))
        ny, nx = r["shape"]
        out = torch.empty((int(r["nz"]), ny, nx), dtype=torch.float32, device=self._device)
        ws = nat.workspace(ws_b.value, self._device)
        zd = self._z_dev()
        ph = r.get("phase")
        nat.check(L.cx_psf_4f(d, spec, nat.ptr(zd), nat.ptr(ph), nat.ptr(out), nat.ptr(ws), ws_b.value,
                              nat.stream_handle(self._device)))
        del keep
        return out if r["zbatch"] else out[0]


    def intensity_to(self, out):
        """PSF stack into ``out``.  For a host (CPU) ``out`` the stack is
        streamed: groups of z-planes are copied to the host on a side stream
        while later groups compute (``cx_psf_4f_to_host``); page-locked memory
        gives the overlap.  ``out`` is valid once the current stream has been
        synchronised."""
        r = self._recipe
        if self.stage != "lens" or self._u is not None or out.is_cuda:
            return super().intensity_to(out)
        torch = nat.torch_mod()
        ny, nx = r["shape"]
        shape = ((int(r["nz"]),) if r["zbatch"] else ()) + (ny, nx)
        if tuple(out.shape) != shape or out.dtype != torch.float32 or not out.is_contiguous():
            raise ValueError(f"out must be a contiguous float32 tensor of shape {shape}")
        L = _sigs(nat.lib())
        d = self._desc()
        spec, keep = self._spec()
        ws_b = nat.c_size_t(0)
        nat.check(L.cx_psf_host_workspace_size(d, spec, ws_b))
        ws = nat.workspace(ws_b.value, self._device)
        cs = nat.copy_stream(self._device)
        ws.record_stream(cs)
        zd = self._z_dev()
        ph = r.get("phase")
        nat.check(L.cx_psf_4f_to_host(d, spec, nat.ptr(zd), nat.ptr(ph), out.data_ptr(), nat.ptr(ws), ws_b.value,
                                      nat.stream_handle(self._device), cs.cuda_stream))
        del keep
        return out


def materialize(field: Field) -> Field:
    """Evaluate a lazy field (no-op for eager fields)."""
    if isinstance(field, LazySourceField):
        return field.materialized()
    return field


def objective_point_source(shape, dx, spectrum, z, f, n, NA, power=1.0, amplitude=1.0, offset=(0.0, 0.0),
                           scalar: bool = True, *, device="cuda", precision=None) -> Field:
    """Point source defocused by ``z`` behind a lens of focal length ``f``
    (functional/sources.py:122-209): ``u = amp (-1j / L^2) exp(-i pi (z/f)
    |r - offset|^2 / L^2)``, ``L^2 = lam f / n``, circular pupil of diameter
    ``2 f NA / n`` and power normalisation.  Evaluated lazily (see module doc)."""
    if not scalar:
        raise NotImplementedError("vectorial fields are not part of this build")
    torch = nat.torch_mod()
    spec = Spectrum.build(spectrum)
    amp = np.asarray(amplitude, dtype=np.float64)
    if amp.size != 1:
        raise AssertionError("scalar fields take a scalar amplitude")
    z_dev = None
    if isinstance(z, torch.Tensor):
        # device-resident z (e.g. a traced/batched argument): read in place
        z_dev = z.detach().reshape(-1).to(device=device, dtype=torch.float64).contiguous()
        nz = int(z_dev.numel())
        z = None
    else:
        z = np.atleast_1d(np.squeeze(np.atleast_1d(np.asarray(z, dtype=np.float64))))
        nz = int(z.size)
    zbatch = nz > 1
    chromatic = not isinstance(spec, MonoSpectrum)
    recipe = dict(shape=(int(shape[0]), int(shape[1])), z=z, z_dev=z_dev, nz=nz, zbatch=zbatch,
                  f=float(f), n=float(n), NA=float(NA), power=None if power is None else float(power),
                  amplitude=float(amp.reshape(())), offset=tuple(float(o) for o in np.broadcast_to(offset, (2,))),
                  src_dx=np.asarray(dx, dtype=np.float64), phase=None, stage="source",
                  precision=precision or config.get_precision())
    dxw = _broadcast_dx(dx, spec.size)
    return LazySourceField(recipe, dxw if chromatic else dxw.reshape(2), spec, chromatic, device)


def plane_wave(shape, dx, spectrum, power=1.0, amplitude=1.0, kykx=(0.0, 0.0), pupil=None, scalar: bool = True,
               *, device="cuda") -> Field:
    """``amp exp(i kykx . r)`` with optional pupil and power normalisation
    (functional/sources.py:212-293), generated on the device by the native
    kernel ``cx_plane_wave``.  Without a pupil |u| is uniform, so the power
    normalisation is analytic (power / (amp^2 N area) folded into the
    amplitude); with a pupil the field's power is measured after it."""
    from .phase_masks import _ew_desc

    torch = nat.torch_mod()
    if not scalar:
        raise NotImplementedError("vectorial plane waves are not part of this build")
    spec = Spectrum.build(spectrum)
    field = Field.empty(shape, dx, spec, device=device)
    amp = float(np.asarray(amplitude).reshape(()))
    ky, kx = (float(v) for v in np.asarray(kykx, dtype=np.float64).reshape(2))
    W = field.n_wv
    dxw = field.dx_wv
    ny, nx = field.spatial_shape
    if power is not None and pupil is None:
        # Field.power (core/field.py:656-661, 728-733): area_w * sum_yx sum_w' density_w' |u|^2
        area = np.prod(dxw, axis=-1)
        dens = np.asarray(spec.density, np.float64) if field.chromatic else np.ones(1)
        p_now = area * (amp * amp) * ny * nx * float(np.sum(dens))
        scale = np.sqrt(float(power) / p_now)
        amps = amp * scale
    else:
        amps = np.full(W, amp)
    tab = nat.upload(np.stack([dxw[:, 0], dxw[:, 1], np.broadcast_to(amps, (W,))], axis=-1), field.device)
    org = np.asarray(field.origin, dtype=np.float64).reshape(-1, 2)[0]
    u = torch.empty(field.u.shape, dtype=torch.complex64, device=field.device)
    nat.check(nat.lib().cx_plane_wave(_ew_desc(field, 0), nat.ptr(tab), ky, kx, float(org[0]), float(org[1]),
                                      nat.ptr(u), nat.stream_handle(u.device)))
    field = field.replace(u=u)
    if pupil is not None:
        field = pupil(field)
        if power is not None:
            pw = field.power
            field = field.replace(u=field.u * torch.sqrt(power / pw))
    return field
