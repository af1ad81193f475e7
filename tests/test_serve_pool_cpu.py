"""Host logic of ToricServerPool: least-loaded routing over per-device
servers, outstanding counts, cancellation and stats, with the device servers
replaced by fakes (no GPU)."""

from __future__ import annotations

from concurrent.futures import Future

import pytest

from generalized_toric_gpu_search_b200.serve import ServeAnswer, ToricServerPool


class FakeServer:
    """Stands in for ToricServer: futures resolve when the test says so."""

    def __init__(self, dev):
        self.dev = dev
        self.futs: list[tuple[Future, list[int], int]] = []
        self.closed = False
        self.pending: list[Future] = []

    def submit(self, indices, td):
        if len(indices) > 15:
            raise ValueError("k too large")
        f = Future()
        self.futs.append((f, list(indices), td))
        self.pending.append(f)
        return f

    def answer_all(self):
        for f, idx, td in self.futs:
            if not f.done():
                f.set_result(ServeAnswer(id=len(idx), max_zeros=49 - td, passed=True,
                                         dedup=False, latency_s=0.0, device_s=0.0))

    def cancel(self, f):
        if f in self.pending and not f.done():
            self.pending.remove(f)
            return f.cancel()
        return False

    def stats(self):
        return {"published": len(self.futs), "finished": sum(f.done() for f, _, _ in self.futs),
                "device_status": 0}

    def close(self):
        self.closed = True


def make_pool(n=3):
    made = {}

    def factory(dev):
        made[dev] = FakeServer(dev)
        return made[dev]

    return ToricServerPool(list(range(n)), factory=factory), made


def test_requests_go_to_the_least_loaded_device():
    pool, made = make_pool(3)
    futs = [pool.submit([1, 2, 3], 10) for _ in range(7)]
    assert [len(made[d].futs) for d in range(3)] == [3, 2, 2]
    assert pool.outstanding() == [3, 2, 2]
    made[1].answer_all()
    assert pool.outstanding() == [3, 0, 2]
    pool.submit([4, 5], 12)
    pool.submit([4, 6], 12)
    assert [len(made[d].futs) for d in range(3)] == [3, 4, 2]
    for d in range(3):
        made[d].answer_all()
    assert pool.outstanding() == [0, 0, 0]
    assert all(f.result().max_zeros == 39 for f in futs)


def test_rejected_submit_does_not_count_and_errors_propagate():
    pool, made = make_pool(2)
    with pytest.raises(ValueError):
        pool.submit(list(range(16)), 10)
    assert pool.outstanding() == [0, 0]
    f = pool.submit([0, 1], 5)
    assert pool.outstanding() == [1, 0]
    made[0].answer_all()
    assert f.result().passed


def test_cancel_reaches_the_owning_device_and_releases():
    pool, made = make_pool(2)
    a = pool.submit([0, 1], 5)
    b = pool.submit([0, 2], 5)
    assert pool.cancel(b)
    assert b.cancelled() and pool.outstanding() == [1, 0]
    assert not pool.cancel(Future())
    made[0].answer_all()
    assert a.result().passed and pool.outstanding() == [0, 0]


def test_stats_sum_devices_and_close_closes_all():
    pool, made = make_pool(2)
    for _ in range(3):
        pool.submit([1], 3)
    made[0].answer_all()
    st = pool.stats()
    assert st["total"]["published"] == 3 and st["total"]["finished"] == 2
    assert set(st["devices"]) == {0, 1}
    with pool:
        pass
    assert all(s.closed for s in made.values())


def test_factory_failure_closes_the_servers_already_built():
    built = []

    def factory(dev):
        if dev == 2:
            raise RuntimeError("no device")
        built.append(FakeServer(dev))
        return built[-1]

    with pytest.raises(RuntimeError):
        ToricServerPool([0, 1, 2], factory=factory)
    assert len(built) == 2 and all(s.closed for s in built)
    with pytest.raises(ValueError):
        ToricServerPool([], factory=factory)
