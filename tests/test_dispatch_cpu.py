"""Multi-device dispatch of a batch (host logic, fake oracles, no GPU)."""

from __future__ import annotations

import threading

from generalized_toric_gpu_search_b200.distance import dispatch_max_zeros_batch


class FakeOracle:
    def __init__(self, dev):
        self.dev = dev
        self.calls = []
        self.threads = set()

    def max_zeros_batch(self, batch, td, sample_count=0, sample_seed=0):
        self.calls.append((len(batch), td, sample_count, sample_seed))
        self.threads.add(threading.get_ident())
        return [100 * self.dev + len(s) for s in batch]


def test_even_chunks_in_order_and_seeds():
    oracles = [FakeOracle(i) for i in range(3)]
    batch = [[0] * (i % 5 + 1) for i in range(10)]
    out = dispatch_max_zeros_batch(oracles, batch, 7, sample_count=50, sample_seed=11)
    assert [c[0] for o in oracles for c in o.calls] == [4, 3, 3]
    assert [o.calls[0][3] for o in oracles] == [11, 11 + 1_000_003, 11 + 2 * 1_000_003]
    want = [100 * 0 + len(s) for s in batch[:4]] + [100 + len(s) for s in batch[4:7]] + \
        [200 + len(s) for s in batch[7:]]
    assert out == want


def test_exact_mode_and_small_batches():
    oracles = [FakeOracle(i) for i in range(4)]
    out = dispatch_max_zeros_batch(oracles, [[1, 2], [3]], 5)
    assert out == [2, 101]
    assert oracles[2].calls == [] and oracles[0].calls == [(1, 5, 0, 0)]
    assert dispatch_max_zeros_batch(oracles, [], 5) == []
    single = FakeOracle(0)
    assert dispatch_max_zeros_batch([single], [[1, 2, 3]], 3, 10, 9) == [3]
    assert single.calls == [(1, 3, 10, 9)]
