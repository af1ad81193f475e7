"""Host logic of ToricBatchServer: canonical dedup and the answer cache.

ToricBatchServer._serve groups a batch by AGL2(F7) canonical mask, evaluates
each group once at its smallest threshold, and answers later requests from a
cache when the cached answer decides their threshold:

  * an exact value (max_zeros <= 49 - td at the evaluated td) decides any td;
  * a failure witness at td_c decides every td >= td_c (d < td_c <= td).

Here the device calls (_canonical, _run) are replaced by the CPU oracle, so
the grouping, cache and answer rules run without a GPU.  Every answer is
checked against the oracle's exact max_zeros under the batch contract:
passed <=> max_zeros <= 49 - td, exact when passed, a witness above 49 - td
otherwise.
"""

from __future__ import annotations

import random
import threading
from concurrent.futures import Future

import numpy as np
import pytest

from generalized_toric_gpu_search_b200.serve import ToricBatchServer
from generalized_toric_gpu_search_b200.tables import N_POINTS, precompute_gl2_perms
from oracle import oracle as orc


@pytest.fixture(scope="module")
def M():
    orc.build()
    return orc.eval_matrix()


def exact(M, s):
    return orc.max_zeros_batch(M, [list(s)], 1)[0]


def agl2_image(s, rng, perms):
    A = perms[rng.randrange(len(perms))]
    da, db = rng.randrange(7), rng.randrange(7)
    img = [int(A[i]) for i in s]
    return sorted(((p // 7 + da) % 7) * 7 + (p % 7 + db) % 7 for p in img)


def make_server(M, cache_size=1 << 20):
    srv = object.__new__(ToricBatchServer)
    srv.dedup = True
    srv.cache_size = cache_size
    srv._cache = {}
    srv._cv = threading.Condition()
    srv._stats = {"published": 0, "finished": 0, "batches": 0, "evaluated": 0,
                  "dedup_answers": 0, "codewords": 0}
    srv.runs = []

    def canonical(masks):
        return orc.canonical_masks(masks)

    def run(sets, tds):
        srv.runs.append(len(sets))
        # the exact value answers any threshold under the batch contract
        return [exact(M, s) for s in sets], 0.0

    srv._canonical = canonical
    srv._run = run
    return srv


def serve(srv, requests):
    batch = []
    for rid, (s, td) in enumerate(requests):
        batch.append((rid, np.asarray(s, dtype=np.int32), int(td), Future(), 0.0))
    srv._serve(batch)
    return [item[3].result(timeout=1) for item in batch]


def check(M, requests, answers):
    for (s, td), a in zip(requests, answers):
        mz = exact(M, s)
        assert a.passed == (mz <= N_POINTS - td)
        if a.passed:
            assert a.max_zeros == mz
        else:
            assert a.max_zeros > N_POINTS - td


def test_equivalent_requests_share_one_evaluation(M):
    rng = random.Random(1)
    perms = precompute_gl2_perms()
    base = sorted(rng.sample(range(N_POINTS), 6))
    d = N_POINTS - exact(M, base)
    requests = [(base, d), (agl2_image(base, rng, perms), d + 1),
                (agl2_image(base, rng, perms), 1)]
    srv = make_server(M)
    answers = serve(srv, requests)
    check(M, requests, answers)
    assert srv.runs == [1]
    assert [a.dedup for a in answers] == [False, True, True]
    assert srv._stats["evaluated"] == 1 and srv._stats["finished"] == 3


def test_cache_decides_later_requests(M):
    rng = random.Random(2)
    perms = precompute_gl2_perms()
    base = sorted(rng.sample(range(N_POINTS), 5))
    d = N_POINTS - exact(M, base)
    srv = make_server(M)
    serve(srv, [(base, 1)])  # exact value cached
    requests = [(agl2_image(base, rng, perms), d), (agl2_image(base, rng, perms), d + 3)]
    answers = serve(srv, requests)
    check(M, requests, answers)
    assert srv.runs == [1]  # the second batch ran nothing
    assert all(a.dedup for a in answers)


def test_cached_failure_decides_only_larger_thresholds(M):
    rng = random.Random(3)
    perms = precompute_gl2_perms()
    base = sorted(rng.sample(range(N_POINTS), 6))
    d = N_POINTS - exact(M, base)
    srv = make_server(M)

    def failing_run(sets, tds):
        srv.runs.append(len(sets))
        out = []
        for s, td in zip(sets, tds):
            mz = exact(M, s)
            # a failure at td reports some witness above 49 - td, here the
            # smallest one allowed
            out.append(mz if mz <= N_POINTS - td else N_POINTS - td + 1)
        return out, 0.0

    srv._run = failing_run
    serve(srv, [(base, d + 2)])  # fails: witness 49 - d - 1 cached at td_c = d + 2
    key = next(iter(srv._cache))
    assert srv._cache[key] == (N_POINTS - d - 1, d + 2)
    later = [(agl2_image(base, rng, perms), d + 4)]  # td >= td_c: decided by the cache
    answers = serve(srv, later)
    check(M, later, answers)
    assert srv.runs == [1] and answers[0].dedup
    lower = [(agl2_image(base, rng, perms), d)]  # td < td_c: must be evaluated
    answers = serve(srv, lower)
    check(M, lower, answers)
    assert srv.runs == [1, 1] and not answers[0].dedup
    assert srv._cache[key] == (N_POINTS - d, d)  # the exact answer replaces the failure


def test_mixed_batch_against_oracle(M):
    rng = random.Random(4)
    perms = precompute_gl2_perms()
    parents = [sorted(rng.sample(range(N_POINTS), rng.randint(3, 6))) for _ in range(6)]
    srv = make_server(M, cache_size=4)
    for _ in range(3):
        requests = []
        for _ in range(12):
            p = parents[rng.randrange(len(parents))]
            s = agl2_image(p, rng, perms) if rng.random() < 0.5 else p
            requests.append((s, rng.randint(1, 40)))
        answers = serve(srv, requests)
        check(M, requests, answers)
        assert len(srv._cache) <= 4
    # repeated or invalid sets keep their own evaluation (no canonical key)
    requests = [([3, 3, 5], 2), ([], 1)]
    answers = serve(srv, requests)
    assert [a.dedup for a in answers] == [False, False]
