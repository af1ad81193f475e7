"""The micro-batching request server (ToricBatchServer) on the B200.

Same contract as the device-resident loop: every served answer equals the
batch oracle's answer for the same (set, threshold) -- the exact max_zeros
when the set passes, a witness above 49 - td when it fails -- whether the
request ran alone, in a batch with others, or was answered from an
equivalent request.
"""

from __future__ import annotations

import random

import pytest

pytestmark = pytest.mark.gpu

N = 49


@pytest.fixture(scope="module")
def server():
    from generalized_toric_gpu_search_b200.serve import ToricBatchServer

    srv = ToricBatchServer(0, k_max=15)
    yield srv
    srv.close()


def same_answer(a, b_mz, td):
    tmax = N - td
    if b_mz <= tmax:
        return a.passed and a.max_zeros == b_mz
    return (not a.passed) and a.max_zeros > tmax


def test_alone_equals_batch(server, gpu_oracle):
    rng = random.Random(4321)
    reqs = [(sorted(rng.sample(range(N), rng.randint(3, 14))), rng.choice([1, 20, 24, 28, 34]))
            for _ in range(80)]
    exact = gpu_oracle.max_zeros_batch([s for s, _ in reqs], 1)
    alone = [server.submit(s, td).result(timeout=120) for s, td in reqs]
    together = server.evaluate(reqs, timeout=300)
    for (s, td), a, t, e in zip(reqs, alone, together, exact):
        assert same_answer(a, e, td), (s, td, a, e)
        assert same_answer(t, e, td), (s, td, t, e)


def test_equivalent_requests_share_one_evaluation(gpu_oracle):
    from generalized_toric_gpu_search_b200.serve import ToricBatchServer
    from generalized_toric_gpu_search_b200.tables import precompute_gl2_perms

    perms = precompute_gl2_perms()
    rng = random.Random(98)
    s = sorted(rng.sample(range(N), 11))
    exact = gpu_oracle.max_zeros_batch([s], 1)[0]
    images = []
    for t in range(6):
        A = perms[rng.randrange(len(perms))]
        images.append(sorted(((int(A[p]) // 7 + t) % 7) * 7 + (int(A[p]) % 7 + 2 * t) % 7
                             for p in s))
    tds = [1, N - exact, N - exact + 1, 30, 1, 45]
    with ToricBatchServer(0, k_max=12) as srv:
        got = srv.evaluate(list(zip(images, tds)), timeout=120)
        st = srv.stats()
    for a, td in zip(got, tds):
        assert same_answer(a, exact, td)
    # one evaluation for the whole class, at the smallest threshold
    assert st["evaluated"] <= st["batches"]
    assert sum(a.dedup for a in got) >= len(got) - st["batches"]


def test_cache_respects_thresholds(server, gpu_oracle):
    rng = random.Random(8)
    s = sorted(rng.sample(range(N), 12))
    exact = gpu_oracle.max_zeros_batch([s], 1)[0]
    strict = server.submit(s, 49).result(timeout=60)
    assert not strict.passed
    # a failure at td = 49 cannot decide a looser request
    loose = server.submit(list(reversed(s)), 1).result(timeout=60)
    assert loose.passed and loose.max_zeros == exact and not loose.dedup
    # the exact value now decides any threshold
    again = server.submit(s, N - exact + 1).result(timeout=60)
    assert again.dedup and not again.passed and again.max_zeros == exact


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


def test_stream_of_mutations(gpu_oracle):
    """A burst of single-point mutations (many equivalent sets) with running
    thresholds, answered exactly as the batch oracle would."""
    from generalized_toric_gpu_search_b200.serve import ToricBatchServer

    rng = random.Random(77)
    parents = [sorted(rng.sample(range(N), rng.randint(10, 13))) for _ in range(12)]
    reqs = []
    for _ in range(300):
        p = list(rng.choice(parents))
        op = rng.randrange(3)
        free = [q for q in range(N) if q not in p]
        if op == 0 and len(p) < 13:
            p.append(rng.choice(free))
        elif op == 1 and len(p) > 10:
            p.remove(rng.choice(p))
        else:
            p[rng.randrange(len(p))] = rng.choice(free)
        reqs.append((sorted(p), rng.choice([1, 22, 25, 27])))
    exact = gpu_oracle.max_zeros_batch([s for s, _ in reqs], 1)
    with ToricBatchServer(0, k_max=13) as srv:
        futs = [srv.submit(s, td) for s, td in reqs]
        got = [f.result(timeout=300) for f in futs]
        st = srv.stats()
    for (s, td), a, e in zip(reqs, got, exact):
        assert same_answer(a, e, td), (s, td, a, e)
    assert st["finished"] == len(reqs) and st["outstanding"] == 0
