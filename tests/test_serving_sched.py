"""Scheduling policy of the continuous-batching server (no GPU): FIFO across
buckets, batch formation, the admission budget."""

import pytest

from chromatix_b200.serving import Request, Scheduler, _prop_bytes, request_bytes


class FakeField:
    def __init__(self, n):
        self.shape = (n, n)


def R(op, n, t, **kw):
    r = Request(op=op, u=FakeField(n), dx=0.3, z=10.0, wavelength=0.5, t_arrival=t, **kw)
    r.id = int(t * 1000)
    return r


def test_oldest_bucket_first_and_batches_by_bucket():
    s = Scheduler(budget_bytes=1e12, max_batch=8)
    for r in [R("asm", 256, 0.001), R("transfer", 256, 0.002), R("asm", 256, 0.003), R("asm", 512, 0.004),
              R("asm", 256, 0.005)]:
        s.add(r)
    b1 = s.pick(1e12)
    assert [r.t_arrival for r in b1] == [0.001, 0.003, 0.005]  # the whole (asm, 256) bucket
    assert [r.op for r in s.pick(1e12)] == ["transfer"]
    assert [r.side for r in s.pick(1e12)] == [512]
    assert s.pick(1e12) is None and len(s) == 0


def test_max_batch_and_czt_singletons():
    s = Scheduler(budget_bytes=1e12, max_batch=3)
    for i in range(7):
        s.add(R("asm", 128, 0.1 + i * 1e-3))
    s.add(R("czt_zoom", 128, 0.05, zoom=2.0))
    s.add(R("czt_zoom", 128, 0.06, zoom=0.5))
    assert [r.op for r in s.pick(1e12)] == ["czt_zoom"]
    assert [r.zoom for r in s.pick(1e12)] == [0.5]
    sizes = []
    while (b := s.pick(1e12)) is not None:
        sizes.append(len(b))
    assert sizes == [3, 3, 1]


def test_admission_budget():
    one = _prop_bytes(1024, 1)
    s = Scheduler(budget_bytes=10 * one, max_batch=32)
    for i in range(6):
        s.add(R("asm", 1024, i * 1e-3))
    # only what fits in the remaining budget is admitted, oldest first
    b = s.pick(budget_left=2.5 * one)
    assert len(b) == 2 and [r.t_arrival for r in b] == [0.0, 0.001]
    assert s.pick(budget_left=0.5 * one) is None  # nothing fits: requests wait
    assert len(s.pick(budget_left=10 * one)) == 4
    with pytest.raises(ValueError):
        s.add(R("asm", 4096, 1.0))  # larger than the whole budget
    assert request_bytes(R("czt_zoom", 256, 0.0)) > 0
