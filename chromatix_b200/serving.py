"""Continuous-batching propagation server.

Requests are independent solves on fields resident in device memory:

  ``"asm"``       ``asm_propagate(field, z, n, pad_width=N/2, mode="same")``
  ``"transfer"``  ``transfer_propagate(field, z, n, pad_width=N/2, mode="same")``
  ``"czt_zoom"``  ``asm_propagate(field, z, n, pad_width=N/2, output_dx=dx/zoom,
                  output_shape=out_shape)`` (the rescaled CZT branch)
  ``"psf"``       the 4f widefield PSF stack of ``objective_point_source`` ->
                  ``phase_change(u)`` -> ``ff_lens`` -> ``.intensity``, with
                  ``u`` the (N, N) float32 phase mask and the optics in
                  ``Request.psf`` (see :class:`Request`)

(functional/propagation.py:168-352, 395-443; functional/sources.py:122-209;
systems/microscopes.py:334-355).  ASM / transfer requests that share
(op, N, n) form a bucket; each scheduler tick launches, per free stream, the
oldest bucket's pending requests as ONE batched ``cx_prop2d_ptrs`` call (per-
request z, wavelength and spacing in the plane table, per-request input /
output pointers), so a batch costs three kernel launches whatever its size.
Those launch sequences are captured once per (stream, bucket, batch size)
into a CUDA graph whose plane table and pointer array live in fixed device
buffers: a later batch of the same shape copies its table from the stream's
page-locked staging buffer into that buffer and replays the graph (two host
calls in place of the three launches and their set-up).  CZT-zoom and PSF requests run one call
sequence each.  Every batch is admitted only while the bytes of the batches
in flight (outputs) plus the streams' workspaces stay under the HBM budget;
requests wait in FIFO order otherwise.  Completion is detected with CUDA
events; latency is host time from arrival to the event.

A request's output does not depend on the batch it ran in, nor on whether
its launch was replayed from a graph: each plane of a batch is transformed
by the same per-row / per-column code as a lone call.  Outputs are
allocated on the server's streams and are complete once the request is
reported done.

The scheduling policy (:class:`Scheduler`) is plain Python over request
metadata, so it is tested without a GPU.
"""

from __future__ import annotations

import collections
import dataclasses
import time

import numpy as np

from . import _native as nat
from . import config

__all__ = ["Request", "Scheduler", "PropagationServer", "percentile", "request_bytes", "batch_cap"]

OPS = ("asm", "transfer", "czt_zoom", "psf")
SINGLETON_OPS = ("czt_zoom", "psf")
# workspace bound of one batched ASM / transfer call: the batch cap per side
# keeps a stream's workspace at or below this size
WS_CAP_BYTES = 1 << 30


@dataclasses.dataclass(eq=False)
class Request:
    """One solve.  ``u``: the (N, N) complex64 field (or, for ``"psf"``, the
    (N, N) float32 phase mask), owned by the client.  ``psf`` (``"psf"``
    only): dict with ``z`` (defocus planes), ``f_obj``, ``f_lens``, ``NA`` and
    optionally ``wavelengths`` / ``density`` (default: ``wavelength`` alone)
    and ``camera_pitch`` (the spacing is then f_lens lambda / (n N pitch), as
    Optical4FSystemPSF.compute_required_spacing gives; else ``dx``)."""

    op: str
    u: object
    dx: float
    z: float
    wavelength: float
    n: float = 1.33
    zoom: float = 1.0
    out_shape: tuple = (512, 512)
    t_arrival: float = 0.0
    psf: dict = None
    id: int = -1
    t_launch: float = float("nan")
    t_done: float = float("nan")
    out: object = None
    ready: object = None  # CUDA event on the client's stream at submit(): the field's writes are complete after it

    @property
    def side(self) -> int:
        return int(self.u.shape[-1])

    @property
    def latency(self) -> float:
        return self.t_done - self.t_arrival

    def bucket(self):
        return (self.op, self.side, float(self.n)) if self.op not in SINGLETON_OPS else (self.op, self.id)


def batch_cap(N: int, max_batch: int) -> int:
    """Largest ASM / transfer batch of side N whose workspace fits WS_CAP_BYTES."""
    return int(max(1, min(max_batch, WS_CAP_BYTES // (32 * N * N))))


def _prop_ws_bytes(N: int, batch: int) -> int:
    """Workspace of one batched ASM/transfer call on the padded (2N x 2N) grid:
    row spectra of the inputs + filtered spectra (mode "same": N output rows)."""
    px = 2 * N
    return 8 * batch * (N * px + N * px) + 512


def _prop_out_bytes(N: int, batch: int) -> int:
    """Outputs (N x N complex64 each) and plane-table bytes of a batch."""
    return 8 * batch * N * N + batch * 64 * 2


def _prop_bytes(N: int, batch: int) -> int:
    """Device bytes one batched ASM/transfer call holds while in flight."""
    return _prop_ws_bytes(N, batch) + _prop_out_bytes(N, batch)


def _czt_out_bytes(out_shape) -> int:
    my, mx = out_shape
    return 8 * my * mx


def _czt_bytes(N: int, out_shape) -> int:
    py = px = 2 * N
    my, mx = out_shape
    return 8 * (2 * py * px + my * px) + 8 * 2 * 8192 + _czt_out_bytes(out_shape)


def _psf_out_bytes(r: Request) -> int:
    nz = int(np.size(r.psf["z"])) if r.psf else 1
    return 4 * nz * r.side * r.side


def _psf_bytes(r: Request) -> int:
    # output stack + the pipeline's L2-sized chunk of row spectra and its tables
    return _psf_out_bytes(r) + (96 << 20) + 16 * r.side * r.side


def request_bytes(r: Request) -> int:
    if r.op == "czt_zoom":
        return _czt_bytes(r.side, r.out_shape)
    if r.op == "psf":
        return _psf_bytes(r)
    return _prop_bytes(r.side, 1)


class Scheduler:
    """FIFO continuous batching with an HBM admission budget.

    ``pick(budget_left)`` returns the next batch to launch: the pending
    requests of the bucket whose oldest request is the oldest overall, up to
    ``batch_cap(N, max_batch)`` and to what the budget admits, or None when
    even its oldest request does not fit (it then waits for batches in
    flight to finish).
    """

    def __init__(self, budget_bytes: float, max_batch: int = 32):
        self.budget = float(budget_bytes)
        self.max_batch = int(max_batch)
        self.queues: dict = collections.OrderedDict()
        self._n = 0

    def add(self, r: Request) -> None:
        if request_bytes(r) > self.budget:
            raise ValueError(f"request needs {request_bytes(r)} bytes, more than the whole budget {self.budget:.0f}")
        self.queues.setdefault(r.bucket(), collections.deque()).append(r)
        self._n += 1

    def __len__(self):
        return self._n

    def pick(self, budget_left: float):
        best, best_t = None, None
        for key, q in self.queues.items():
            if q and (best_t is None or q[0].t_arrival < best_t):
                best, best_t = key, q[0].t_arrival
        if best is None:
            return None
        q = self.queues[best]
        if best[0] in SINGLETON_OPS:
            if request_bytes(q[0]) > budget_left:
                return None
            batch = [q.popleft()]
        else:
            N = best[1]
            k = 0
            while k < min(len(q), batch_cap(N, self.max_batch)) and _prop_bytes(N, k + 1) <= budget_left:
                k += 1
            if k == 0:
                return None
            batch = [q.popleft() for _ in range(k)]
        if not q:
            del self.queues[best]
        self._n -= len(batch)
        return batch


def percentile(values, p):
    v = np.sort(np.asarray(values, dtype=np.float64))
    if v.size == 0:
        return float("nan")
    return float(np.percentile(v, p))


class _Slot:
    """A stream with its page-locked staging buffer and fixed device buffer for
    plane tables and pointers, its workspace and its captured launch graphs."""

    def __init__(self, torch, device, staging_bytes):
        self.stream = torch.cuda.Stream(device=device)
        self.pinned = torch.empty(staging_bytes, dtype=torch.uint8).pin_memory()
        self.dev = torch.empty(staging_bytes, dtype=torch.uint8, device=device)
        self.busy = None  # (event, batch, bytes, keepalive) of the batch in flight
        self.ws = None  # workspace, grown to the largest batch this stream has run
        self.graphs = {}  # (op, N, n, batch, workspace address) -> CUDA graph of the batched launch
        self._torch = torch
        self._device = device

    def workspace(self, nbytes: int, reserve: int = 0):
        """At least ``nbytes``; a regrowth allocates ``reserve`` bytes at once
        (the largest batch of that shape), so a stream regrows at most once
        per request shape instead of on every larger batch.  Graphs captured
        with the old workspace are dropped."""
        if self.ws is None or self.ws.numel() < nbytes:
            self.ws = None
            self.graphs.clear()
            self.ws = self._torch.empty(max(int(nbytes), int(reserve), 256), dtype=self._torch.uint8,
                                        device=self._device)
        return self.ws


class PropagationServer:
    """Continuous-batching server on one device (one per GPU; replicas scale out).

    ``use_graphs``: replay the batched ASM / transfer launches from CUDA
    graphs (captured on first use per stream and batch shape, or ahead of
    time by :meth:`warmup`)."""

    def __init__(self, device="cuda", budget_bytes: float = 60e9, n_streams: int = 4, max_batch: int = 32,
                 precision=None, use_graphs: bool = True):
        torch = nat.torch_mod()
        self.torch = torch
        self.device = torch.device(device)
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.sched = Scheduler(budget_bytes, max_batch)
        self.max_batch = int(max_batch)
        self.precision = precision or config.get_precision()
        self.use_graphs = bool(use_graphs)
        staging = self.max_batch * (nat.PLANE_DTYPE.itemsize + 16) + 256
        self.slots = [_Slot(torch, self.device, staging) for _ in range(int(n_streams))]
        self.inflight_bytes = 0
        self.completed: list = []
        self._next_id = 0
        # per-op totals: host seconds spent launching, device ms between the
        # batch's first and last kernel (streams overlap, so these can exceed
        # wall time), batches; graph replays and captures
        self.host_s = collections.Counter()
        self.gpu_ms = collections.Counter()
        self.batches = collections.Counter()
        self.graph_replays = 0
        self.graph_captures = 0
        L = nat.lib()
        if not hasattr(L, "_cx_prop2d_ptrs_sig"):
            L.cx_prop2d_ptrs.restype = nat.c_int32
            L.cx_prop2d_ptrs.argtypes = [nat.ctypes.POINTER(nat.cx_prop2d_desc), nat.c_void_p, nat.c_void_p,
                                         nat.c_void_p, nat.c_void_p, nat.c_void_p, nat.c_size_t, nat.c_void_p]
            L.cx_init.restype = nat.c_int32
            L._cx_prop2d_ptrs_sig = True
        self.L = L
        with torch.cuda.device(self.device):
            nat.check(L.cx_init())  # twiddle tables uploaded before any capture

    # -- client side ------------------------------------------------------------
    def submit(self, r: Request) -> Request:
        if r.op not in OPS:
            raise ValueError(f"unknown op {r.op!r}; expected one of {OPS}")
        u = r.u
        if r.op == "psf":
            if not (u.is_cuda and u.dtype == self.torch.float32 and u.ndim == 2 and u.shape[0] == u.shape[1]):
                raise ValueError("a PSF request's phase mask is a square (N, N) float32 CUDA tensor")
            if not r.psf or "z" not in r.psf:
                raise ValueError("a PSF request needs psf={'z': ..., 'f_obj': ..., 'f_lens': ..., 'NA': ...}")
        elif not (u.is_cuda and u.dtype == self.torch.complex64 and u.ndim == 2 and u.shape[0] == u.shape[1]
                  and u.is_contiguous()):
            raise ValueError("a request field is a contiguous square (N, N) complex64 CUDA tensor")
        if not r.t_arrival:
            r.t_arrival = time.perf_counter()
        # the field may still be in flight on the client's stream (written by an
        # asynchronous kernel or copy); the server's stream waits for this event
        # before its first kernel reads it
        r.ready = self.torch.cuda.Event()
        r.ready.record(self.torch.cuda.current_stream(u.device))
        r.id = self._next_id
        self._next_id += 1
        self.sched.add(r)
        return r

    @property
    def busy(self) -> bool:
        return len(self.sched) > 0 or any(s.busy is not None for s in self.slots)

    # -- scheduler tick -----------------------------------------------------------
    def step(self) -> list:
        """Retire finished batches, launch new ones on free streams; returns
        the requests completed in this tick."""
        done = self._retire()
        for slot in self.slots:
            if slot.busy is not None:
                continue
            # workspaces stay allocated between batches: every other stream's
            # held workspace counts against the budget; this stream's own is
            # reused (or replaced) by the batch it launches
            left = self.sched.budget - self.inflight_bytes - self.held_workspace_bytes(exclude=slot)
            batch = self.sched.pick(left)
            if batch is None:
                continue  # another free stream may hold the workspace this batch needs
            self._launch(slot, batch, left)
        return done

    def held_workspace_bytes(self, exclude=None) -> int:
        """Device bytes of the streams' workspaces (kept between batches)."""
        return sum(s.ws.numel() for s in self.slots if s is not exclude and s.ws is not None)

    def drain(self) -> list:
        out = []
        while self.busy:
            out += self.step()
        return out

    def warmup(self, ops=("asm", "transfer"), sides=(256, 512, 1024, 2048), n: float = 1.33) -> None:
        """Capture the batched launch graphs of every (op, side, batch size) on
        every stream ahead of a request stream (a capture launches nothing).
        Each stream's workspace is sized first for the largest of them, so the
        graphs stay valid."""
        if not self.use_graphs:
            return
        need = max(_prop_ws_bytes(N, batch_cap(N, self.max_batch)) for N in sides)
        for slot in self.slots:
            slot.workspace(need)
        for slot in self.slots:
            for op in ops:
                for N in sides:
                    for B in range(1, batch_cap(N, self.max_batch) + 1):
                        d, wsb = self._prop_desc(op, N, n, B)
                        self._graph(slot, (op, N, float(n), B), d, wsb)
        # grow each stream's allocator pool to a full batch of outputs per
        # side now: a fresh cudaMalloc inside a stream's first large batches
        # stalls the scheduler for tens of milliseconds
        torch = self.torch
        for slot in self.slots:
            with torch.cuda.stream(slot.stream):
                held = [torch.empty((N, N), dtype=torch.complex64, device=self.device)
                        for N in sides for _ in range(batch_cap(N, self.max_batch))]
                del held
        self.torch.cuda.synchronize(self.device)

    def _retire(self) -> list:
        done = []
        for slot in self.slots:
            if slot.busy is None:
                continue
            ev, batch, nbytes, keep = slot.busy
            if not ev.query():
                continue
            t = time.perf_counter()
            self.gpu_ms[batch[0].op] += keep[0].elapsed_time(ev)
            for r in batch:
                r.t_done = t
            self.inflight_bytes -= nbytes
            slot.busy = None
            done += batch
        self.completed += done
        return done

    def _launch(self, slot: _Slot, batch: list, budget_left: float = float("inf")) -> None:
        torch = self.torch
        t = time.perf_counter()
        for r in batch:
            r.t_launch = t
        for r in batch:
            if r.ready is not None:
                slot.stream.wait_event(r.ready)
        op = batch[0].op
        with torch.cuda.stream(slot.stream):
            # recorded just before the batch's kernels are issued (device time only)
            slot.ev0 = ev0 = torch.cuda.Event(enable_timing=True)
            if op == "czt_zoom":
                nbytes = _czt_out_bytes(batch[0].out_shape)
                keep = self._run_czt(slot, batch[0])
            elif op == "psf":
                nbytes = _psf_out_bytes(batch[0])
                keep = self._run_psf(slot, batch[0])
            else:
                nbytes = _prop_out_bytes(batch[0].side, len(batch))
                keep = self._run_prop(slot, batch, budget_left - nbytes)
            ev = torch.cuda.Event(enable_timing=True)
            ev.record(slot.stream)
        self.inflight_bytes += nbytes
        slot.busy = (ev, batch, nbytes, (ev0, keep))
        self.host_s[op] += time.perf_counter() - t
        self.batches[op] += 1

    def _prop_desc(self, op, N, n, B):
        d = nat.cx_prop2d_desc()
        d.ny = d.nx = N
        d.pad_y = d.pad_x = N // 2
        d.n_wv = 1
        d.n_in_planes = d.n_out_planes = B
        d.mode_same = 1
        d.kernel = nat.CX_KERNEL_ASM if op == "asm" else nat.CX_KERNEL_TRANSFER
        d.precision = config.precision_code(self.precision, tensor_core=config.tensor_core_grid(2 * N, 2 * N))
        d.n_medium = float(n)
        wsb = nat.c_size_t(0)
        nat.check(self.L.cx_prop2d_workspace_size(d, wsb))
        return d, wsb.value

    @staticmethod
    def _table_bytes(B: int):
        """(offset of the pointer array, bytes to upload) of a B-request table."""
        off_p = (B * nat.PLANE_DTYPE.itemsize + 15) // 16 * 16
        return off_p, off_p + 16 * B

    def _call_prop(self, slot: _Slot, d, wsb: int, B: int) -> None:
        """``cx_prop2d_ptrs`` on the stream's fixed table buffer (current stream)."""
        off_p, _ = self._table_bytes(B)
        base = slot.dev.data_ptr()
        nat.check(self.L.cx_prop2d_ptrs(d, base, base + off_p, base + off_p + 8 * B, None, slot.ws.data_ptr(), wsb,
                                        self.torch.cuda.current_stream(self.device).cuda_stream))

    def _graph(self, slot: _Slot, key, d, wsb: int):
        """The captured launch sequence of ``key`` on this stream (captured on
        first use): the three kernels of ``cx_prop2d_ptrs`` reading the plane
        table and pointers from the stream's fixed device buffer."""
        torch = self.torch
        gkey = key + (slot.ws.data_ptr(),)
        g = slot.graphs.get(gkey)
        if g is None:
            g = torch.cuda.CUDAGraph()
            with torch.cuda.stream(slot.stream):
                g.capture_begin(capture_error_mode="thread_local")
                try:
                    self._call_prop(slot, d, wsb, key[3])
                finally:
                    g.capture_end()
            slot.graphs[gkey] = g
            self.graph_captures += 1
        return g

    def _run_prop(self, slot: _Slot, batch: list, ws_budget: float = float("inf")):
        torch = self.torch
        N = batch[0].side
        B = len(batch)
        planes = np.zeros(B, dtype=nat.PLANE_DTYPE)
        planes["z"] = [r.z for r in batch]
        planes["wavelength"] = [r.wavelength for r in batch]
        planes["dy"] = planes["dx"] = [r.dx for r in batch]
        planes["in_plane"] = np.arange(B)
        for r in batch:
            r.out = torch.empty((N, N), dtype=torch.complex64, device=self.device)
        ptrs = np.array([r.u.data_ptr() for r in batch] + [r.out.data_ptr() for r in batch], dtype=np.uint64)
        pb = planes.view(np.uint8)
        off_p, n_up = self._table_bytes(B)
        host = slot.pinned.numpy()
        host[: pb.size] = pb
        host[off_p: off_p + ptrs.nbytes] = ptrs.view(np.uint8)
        op, n = batch[0].op, float(batch[0].n)
        d, wsb = self._prop_desc(op, N, n, B)
        # grow once to the largest batch of this shape, as far as the budget allows
        reserve = min(_prop_ws_bytes(N, batch_cap(N, self.max_batch)), max(ws_budget, wsb))
        slot.workspace(wsb, reserve=reserve)
        g = self._graph(slot, (op, N, n, B), d, wsb) if self.use_graphs else None
        slot.ev0.record(slot.stream)
        # this batch's table: staging buffer -> the stream's fixed device buffer
        # (asynchronous; the staging buffer is reused only after the batch retires)
        slot.dev[:n_up].copy_(slot.pinned[:n_up], non_blocking=True)
        if g is not None:
            g.replay()
            self.graph_replays += 1
        else:
            self._call_prop(slot, d, wsb, B)
        for r in batch:
            r.u.record_stream(slot.stream)
        return None

    def _run_czt(self, slot: _Slot, r: Request):
        """``asm_propagate(..., output_dx=dx/zoom, output_shape=out_shape)`` as
        one ``cx_czt_propagate`` call (the path the functional API takes)."""
        from .functional.rescaled import _czt_prop_sigs, cx_czt_prop_desc

        torch = self.torch
        L = _czt_prop_sigs(self.L)
        N = r.side
        d = cx_czt_prop_desc()
        d.ny = d.nx = N
        d.pad_y = d.pad_x = N // 2
        d.my, d.mx = int(r.out_shape[0]), int(r.out_shape[1])
        d.n_fields = 1
        d.kernel = nat.CX_KERNEL_ASM
        d.precision = config.precision_code(self.precision)
        d.n_medium, d.z, d.wavelength = float(r.n), float(r.z), float(r.wavelength)
        d.dy_in = d.dx_in = float(r.dx)
        d.dy_out = d.dx_out = float(np.array([r.dx / r.zoom] * 2)[0])
        wsb = nat.c_size_t(0)
        nat.check(L.cx_czt_propagate_workspace_size(d, wsb))
        ws = slot.workspace(wsb.value)
        r.out = torch.empty((d.my, d.mx), dtype=torch.complex64, device=self.device)
        slot.ev0.record(slot.stream)
        nat.check(L.cx_czt_propagate(d, r.u.data_ptr(), r.out.data_ptr(), ws.data_ptr(), wsb.value,
                                     slot.stream.cuda_stream))
        r.u.record_stream(slot.stream)
        return None

    def _run_psf(self, slot: _Slot, r: Request):
        """The fused PSF pipeline (one ``cx_psf_4f`` call) through the
        functional API, on this stream."""
        from . import functional as cf

        p = r.psf
        N = r.side
        lam = np.atleast_1d(np.asarray(p.get("wavelengths", r.wavelength), dtype=np.float64))
        dens = np.asarray(p.get("density", np.ones(lam.size)), dtype=np.float64)
        f_lens = float(p["f_lens"])
        if "camera_pitch" in p:
            dxw = f_lens * lam / (float(r.n) * N * float(p["camera_pitch"]))
            dx = np.stack([dxw, dxw], -1) if lam.size > 1 else float(dxw[0])
        else:
            dx = r.dx
        spec = (lam, dens) if lam.size > 1 else float(lam[0])
        slot.ev0.record(slot.stream)
        f = cf.objective_point_source((N, N), dx, spec, np.asarray(p["z"], dtype=np.float64), float(p["f_obj"]),
                                      float(r.n), float(p["NA"]), device=self.device)
        f = cf.ff_lens(cf.phase_change(f, r.u), f_lens, float(r.n))
        r.out = f.intensity
        r.u.record_stream(slot.stream)
        return None
