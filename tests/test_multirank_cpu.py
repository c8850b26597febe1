"""The N > 1 path on CPU: world_size-2 gloo ranks (127.0.0.1) agree on the
maximum of their timings, as bench.py reports it, and the replicas' work
units do not depend on the rank count."""

import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench

        got = bench.max_over_ranks([1.0 + rank, 10.0 - rank], dist, "cpu")
        q.put((rank, got))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_max_over_ranks_gloo_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=90) for _ in procs)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    assert res[0] == res[1] == [2.0, 10.0]


def test_max_over_ranks_single_process():
    import bench

    assert bench.max_over_ranks([3.0, 4.0]) == [3.0, 4.0]
