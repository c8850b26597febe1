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


def test_gpus_flag_launches_one_rank_per_gpu(monkeypatch):
    """``bench.py --gpus N`` outside a launcher starts N ranks through
    torch.distributed.run on 127.0.0.1 with the same arguments, and exits
    with the launcher's status."""
    import sys

    import bench

    calls = []
    monkeypatch.setattr(bench.subprocess, "call", lambda cmd: calls.append(cmd) or 7)
    monkeypatch.delenv("WORLD_SIZE", raising=False)
    monkeypatch.setattr(sys, "argv", ["bench.py", "--gpus", "4", "--steps", "3", "--warmup", "3"])
    with pytest.raises(SystemExit) as ex:
        bench.main()
    assert ex.value.code == 7
    (cmd,) = calls
    assert cmd[1:3] == ["-m", "torch.distributed.run"]
    assert "--nproc-per-node=4" in cmd and "--nnodes=1" in cmd
    assert cmd[cmd.index("--master-addr") + 1] == "127.0.0.1"
    assert cmd[-6:] == ["--gpus", "4", "--steps", "3", "--warmup", "3"]
    assert cmd[-7].endswith("bench.py")
