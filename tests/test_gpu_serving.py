"""Continuous-batching server on the GPU: every request's result is identical
(bit for bit) to the same propagation issued alone through the functional
API, whatever batch it ran in; the admission budget holds."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _field(n, seed):
    import torch

    rng = np.random.default_rng(seed)
    u = np.exp(1j * rng.uniform(0, 2 * np.pi, (n, n))).astype(np.complex64)
    return torch.as_tensor(u, device="cuda")


def _alone(r):
    import chromatix_b200.functional as cf
    from chromatix_b200.core.field import Field

    f = Field.build(r.u, r.dx, r.wavelength)
    N = r.side
    if r.op == "asm":
        return cf.asm_propagate(f, r.z, r.n, N // 2, mode="same").u
    if r.op == "transfer":
        return cf.transfer_propagate(f, r.z, r.n, N // 2, mode="same").u
    return cf.asm_propagate(f, r.z, r.n, N // 2, output_dx=np.array([r.dx / r.zoom] * 2), output_shape=r.out_shape).u


def test_mixed_requests_match_lone_calls():
    import torch

    from chromatix_b200.serving import PropagationServer, Request

    rng = np.random.default_rng(0)
    sides = [64, 128, 256]
    fields = {n: [_field(n, 10 * n + k) for k in range(3)] for n in sides}
    srv = PropagationServer(budget_bytes=4e9, n_streams=3, max_batch=8)
    reqs = []
    for i in range(60):
        n = int(rng.choice(sides))
        op = ["asm", "transfer", "czt_zoom"][int(rng.integers(0, 3))]
        r = Request(op=op, u=fields[n][int(rng.integers(0, 3))], dx=0.3, z=float(rng.uniform(1, 500)),
                    wavelength=float(rng.uniform(0.4, 0.7)), zoom=float(rng.uniform(0.25, 4)), out_shape=(64, 64))
        reqs.append(srv.submit(r))
        if i % 7 == 0:
            srv.step()
    srv.drain()
    torch.cuda.synchronize()
    assert len(srv.completed) == 60
    assert srv.inflight_bytes == 0
    batched = [r for r in reqs if r.op != "czt_zoom"]
    assert any(r.t_launch == s.t_launch for r in batched for s in batched if r is not s)  # some ran together
    for r in reqs:
        ref = _alone(r)
        torch.cuda.synchronize()
        assert r.out.shape == ref.shape
        assert torch.equal(r.out, ref), (r.op, r.side)
        assert r.latency >= 0


def test_budget_limits_batches():
    import torch

    from chromatix_b200.serving import PropagationServer, Request, _prop_bytes

    u = _field(256, 1)
    srv = PropagationServer(budget_bytes=2.5 * _prop_bytes(256, 1), n_streams=4, max_batch=16)
    reqs = [srv.submit(Request(op="asm", u=u, dx=0.3, z=10.0 + i, wavelength=0.5)) for i in range(6)]
    peak = 0
    while srv.busy:
        srv.step()
        peak = max(peak, srv.inflight_bytes + srv.held_workspace_bytes())
    torch.cuda.synchronize()
    assert peak <= srv.sched.budget
    for r in reqs:
        assert torch.equal(r.out, _alone(r))


def test_request_written_on_a_producer_stream_is_read_after_its_writes():
    """A field still being written on the client's stream when it is submitted
    (no synchronisation in between) is read only after those writes: the
    server's stream waits on an event recorded at submit()."""
    import torch

    from chromatix_b200.serving import PropagationServer, Request

    src = _field(512, 5)
    u = torch.zeros_like(src)
    producer = torch.cuda.Stream()
    srv = PropagationServer(budget_bytes=4e9, n_streams=2, max_batch=4)
    torch.cuda.synchronize()
    with torch.cuda.stream(producer):
        torch.cuda._sleep(50_000_000)  # tens of milliseconds of device time before the write lands
        u.copy_(src)
        r = srv.submit(Request(op="asm", u=u, dx=0.3, z=50.0, wavelength=0.5))
    srv.drain()
    torch.cuda.synchronize()
    ref = _alone(Request(op="asm", u=src, dx=0.3, z=50.0, wavelength=0.5))
    torch.cuda.synchronize()
    assert torch.equal(r.out, ref)


def _psf_request(rng, N):
    import torch

    from chromatix_b200.serving import Request

    ph = torch.as_tensor(rng.uniform(0, 2 * np.pi, (N, N)).astype(np.float32), device="cuda")
    z = np.sort(rng.uniform(-3, 3, 4))
    return Request(op="psf", u=ph, dx=0.0, z=0.0, wavelength=0.532,
                   psf={"z": z, "f_obj": 8000.0, "f_lens": 200000.0, "NA": 0.6, "camera_pitch": 6.5,
                        "wavelengths": [0.45, 0.532, 0.63]})


def _psf_alone(r):
    import chromatix_b200.functional as cf

    p = r.psf
    N = r.side
    lam = np.asarray(p["wavelengths"])
    dxw = p["f_lens"] * lam / (r.n * N * p["camera_pitch"])
    f = cf.objective_point_source((N, N), np.stack([dxw, dxw], -1), (lam, np.ones(lam.size)), p["z"], p["f_obj"],
                                  r.n, p["NA"])
    return cf.ff_lens(cf.phase_change(f, r.u), p["f_lens"], r.n).intensity


def test_graph_replay_and_psf_requests_match_lone_calls():
    """Batched launches replayed from captured CUDA graphs give the same bits
    as the eager launch path and as lone calls; PSF requests in the mix give
    the lone fused PSF's bits."""
    import torch

    from chromatix_b200.serving import PropagationServer, Request

    rng = np.random.default_rng(3)
    fields = {n: [_field(n, 7 * n + k) for k in range(2)] for n in (128, 256)}
    specs = []
    for i in range(40):
        n = (128, 256)[i % 2]
        op = ("asm", "transfer", "czt_zoom", "psf")[i % 4] if i % 5 else "asm"
        specs.append((op, n, int(rng.integers(0, 2)), float(rng.uniform(1, 500)), float(rng.uniform(0.4, 0.7)),
                      float(rng.uniform(0.25, 4))))
    psf_reqs = {i: _psf_request(np.random.default_rng(100 + i), 256) for i in range(40) if specs[i][0] == "psf"}
    outs = {}
    for graphs in (True, False):
        srv = PropagationServer(budget_bytes=8e9, n_streams=3, max_batch=8, use_graphs=graphs)
        if graphs:
            srv.warmup(ops=("asm", "transfer"), sides=(128, 256))
            assert srv.graph_captures > 0
        reqs = []
        for i, (op, n, k, z, lam, zoom) in enumerate(specs):
            if op == "psf":
                r0 = psf_reqs[i]
                r = Request(op="psf", u=r0.u, dx=0.0, z=0.0, wavelength=0.532, psf=r0.psf)
            else:
                r = Request(op=op, u=fields[n][k], dx=0.3, z=z, wavelength=lam, zoom=zoom, out_shape=(64, 64))
            reqs.append(srv.submit(r))
            if i % 6 == 0:
                srv.step()
        srv.drain()
        torch.cuda.synchronize()
        if graphs:
            assert srv.graph_replays > 0
        outs[graphs] = [r.out for r in reqs]
        for r in reqs:
            ref = _psf_alone(r) if r.op == "psf" else _alone(r)
            torch.cuda.synchronize()
            assert torch.equal(r.out, ref), (r.op, r.side, graphs)
    for a, b in zip(outs[True], outs[False]):
        assert torch.equal(a, b)
