"""The device-resident request loop (ToricServer) on the B200.

Contract under test: every served answer equals the batch oracle's answer for
the same (set, threshold) -- the exact max_zeros when the set passes, a
witness above 49 - td when it fails -- whether the request ran alone or in a
mix with other requests arriving while it was on the GPU.
"""

from __future__ import annotations

import random

import pytest

pytestmark = pytest.mark.gpu

N = 49


@pytest.fixture(scope="module")
def server():
    from generalized_toric_gpu_search_b200.serve import ToricServer

    srv = ToricServer(0, k_max=15, max_slots=256, idle_us=3000, life_ms=100)
    yield srv
    srv.close()


def same_answer(a, b_mz, td):
    tmax = N - td
    if b_mz <= tmax:
        return a.passed and a.max_zeros == b_mz
    return (not a.passed) and a.max_zeros > tmax


def test_alone_equals_mix_equals_batch(server, gpu_oracle):
    """Requests of the served stream's sizes (k = 10..15, thresholds around
    the best-known distances) give the batch oracle's answer alone and when
    interleaved with 200 others in flight together."""
    rng = random.Random(1234)
    reqs = []
    for _ in range(60):
        k = rng.randint(10, 15)
        reqs.append((sorted(rng.sample(range(N), k)), rng.choice([1, 18, 21, 24, 26, 28])))
    exact = gpu_oracle.max_zeros_batch([s for s, _ in reqs], 1)
    alone = [server.submit(s, td).result(timeout=120) for s, td in reqs]
    # the same requests interleaved with 200 unrelated ones, all in flight together
    noise = [(sorted(rng.sample(range(N), rng.randint(3, 15))), rng.randint(1, 30))
             for _ in range(200)]
    mixed_reqs, mine_at = [], []
    for i, r in enumerate(reqs):
        mine_at.append(len(mixed_reqs))
        mixed_reqs.append(r)
        mixed_reqs.extend(noise[4 * i: 4 * i + 4])
    futs = [server.submit(s, td) for s, td in mixed_reqs]
    mixed = [f.result(timeout=300) for f in futs]
    mixed_mine = [mixed[j] for j in mine_at]
    for (s, td), a, m, e in zip(reqs, alone, mixed_mine, exact):
        assert same_answer(a, e, td), (s, td, a, e)
        assert same_answer(m, e, td), (s, td, m, e)
        if a.passed:
            assert a.max_zeros == m.max_zeros == e


def test_dedup_by_canonical_form(server, gpu_oracle):
    from generalized_toric_gpu_search_b200.tables import precompute_gl2_perms

    perms = precompute_gl2_perms()
    rng = random.Random(99)
    s = sorted(rng.sample(range(N), 9))
    exact = gpu_oracle.max_zeros_batch([s], 1)[0]
    first = server.submit(s, 1).result(timeout=60)
    assert first.passed and first.max_zeros == exact
    A = perms[517]
    image = sorted(((int(A[p]) // 7 + 3) % 7) * 7 + (int(A[p]) % 7 + 5) % 7 for p in s)
    second = server.submit(image, 1).result(timeout=60)
    assert second.dedup and second.passed and second.max_zeros == exact
    # a stricter threshold is decided by the stored exact value too
    td = N - exact + 1
    third = server.submit(s, td).result(timeout=60)
    assert third.dedup and not third.passed and third.max_zeros == exact


def test_dedup_respects_thresholds(server, gpu_oracle):
    rng = random.Random(7)
    s = sorted(rng.sample(range(N), 8))
    exact = gpu_oracle.max_zeros_batch([s], 1)[0]
    # the first request fails early against an impossible threshold ...
    strict = server.submit(s, 49).result(timeout=60)
    assert not strict.passed
    # ... which cannot decide a looser request unless its witness does
    loose = server.submit(list(reversed(s)), 1).result(timeout=60)
    assert loose.passed and loose.max_zeros == exact


def test_admission_beyond_slots(gpu_oracle):
    from generalized_toric_gpu_search_b200.serve import ToricServer

    rng = random.Random(5)
    reqs = [(sorted(rng.sample(range(N), rng.randint(4, 9))), 1) for _ in range(150)]
    exact = gpu_oracle.max_zeros_batch([s for s, _ in reqs], 1)
    with ToricServer(0, k_max=12, max_slots=4, table_capacity=-1) as srv:
        assert srv.slots == 4
        got = srv.evaluate(reqs, timeout=300)
        st = srv.stats()
    assert [a.max_zeros for a in got] == exact
    assert all(a.passed and not a.dedup for a in got)
    assert st["finished"] == 150 and st["outstanding"] == 0


def test_edge_requests(server):
    assert server.submit([], 5).result(timeout=30).max_zeros == 0
    one = server.submit([17], 1).result(timeout=30)
    assert one.passed and one.max_zeros == 0
    dup = server.submit([3, 9, 3], 1).result(timeout=30)
    assert not dup.passed and dup.max_zeros == 49
    with pytest.raises(ValueError):
        server.submit(list(range(16)), 1)
    with pytest.raises(ValueError):
        server.submit([0, 49], 1)


def test_loop_relaunches_after_idle(gpu_oracle):
    import time

    from generalized_toric_gpu_search_b200.serve import ToricServer

    rng = random.Random(3)
    with ToricServer(0, k_max=10, max_slots=32, idle_us=500, life_ms=50) as srv:
        a = srv.submit(sorted(rng.sample(range(N), 7)), 1).result(timeout=60)
        time.sleep(0.3)  # the loop exits after 0.5 ms idle
        s2 = sorted(rng.sample(range(N), 8))
        b = srv.submit(s2, 1).result(timeout=60)
        st = srv.stats()
    assert a.passed and b.passed
    assert b.max_zeros == gpu_oracle.max_zeros_batch([s2], 1)[0]
    assert st["loop_launches"] >= 2


def test_pool_of_every_visible_device_matches_batch(gpu_oracle):
    """ToricServerPool over the visible GPUs (one here): each device runs its
    own request loop, and the answers equal the batch oracle's."""
    import torch

    from generalized_toric_gpu_search_b200.serve import ToricServerPool

    rng = random.Random(77)
    reqs = [(sorted(rng.sample(range(N), rng.randint(8, 13))), rng.choice([1, 20, 24]))
            for _ in range(24)]
    exact = gpu_oracle.max_zeros_batch([s for s, _ in reqs], 1)
    with ToricServerPool(k_max=13, max_slots=64, idle_us=3000, life_ms=100) as pool:
        assert len(pool.servers) == torch.cuda.device_count()
        got = pool.evaluate(reqs, timeout=300)
        # done callbacks run in the servers' pump threads, just after the
        # answers are delivered
        import time

        t_end = time.time() + 5.0
        while any(pool.outstanding()) and time.time() < t_end:
            time.sleep(0.01)
        assert pool.outstanding() == [0] * len(pool.servers)
        assert pool.stats()["total"]["finished"] == len(reqs)
    for (s, td), a, e in zip(reqs, got, exact):
        assert same_answer(a, e, td), (s, td, a, e)
