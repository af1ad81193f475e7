"""Information-set (Brouwer-Zimmermann) enumeration against the oracle and
against the independent orbit enumeration.

Same contract as every exact mode: a passing set returns exactly max_zeros, a
failing set returns a value > 49 - td.
"""

from __future__ import annotations

import random

import numpy as np
import pytest

from oracle import oracle as orc

pytestmark = pytest.mark.gpu

N = 49
INFOSET = 3
ORBIT = 2


def rand_sets(rng, n, kmin, kmax):
    return [sorted(rng.sample(range(N), rng.randint(kmin, kmax))) for _ in range(n)]


def check_decisions(got, exact, tds):
    for g, e, td in zip(got, exact, tds):
        tmax = N - td
        if e <= tmax:
            assert g == e
        else:
            assert g > tmax


def oracle_for(M, enumeration, **kw):
    from generalized_toric_gpu_search_b200.distance import DistanceOracleCUDABP, LaunchConfig

    return DistanceOracleCUDABP(0, M, LaunchConfig(enumeration=enumeration, **kw), autotune=False)


@pytest.fixture(scope="module")
def infoset(M):
    return oracle_for(M, INFOSET)


@pytest.fixture(scope="module")
def orbit(M):
    return oracle_for(M, ORBIT)


def test_known_answers(infoset, golden):
    sets = [k["set"] for k in golden["max_zeros_kats"]]
    want = [k["max_zeros"] for k in golden["max_zeros_kats"]]
    assert infoset.max_zeros_batch(sets, 1) == want
    assert infoset.min_distance([0, 8, 18, 23, 30, 39, 43]) == 34
    assert infoset.min_distance([1, 6, 7, 16, 19, 37, 40, 42]) == 24


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_mixed_k_exact_against_oracle(M, infoset, seed):
    rng = random.Random(300 + seed)
    sets = rand_sets(rng, 80, 1, 8)
    assert infoset.max_zeros_batch(sets, 1) == orc.max_zeros_batch(M, sets, 1)


def test_threshold_decisions(M, infoset):
    rng = random.Random(301)
    sets = rand_sets(rng, 150, 2, 8)
    exact = orc.max_zeros_batch(M, sets, 1)
    tds = [rng.randint(1, 49) for _ in sets]
    check_decisions(infoset.max_zeros_batch(sets, tds), exact, tds)
    for td in (10, 20, 30, 40):
        check_decisions(infoset.max_zeros_batch(sets, td), exact, [td] * len(sets))


def test_edge_cases(M, infoset):
    assert infoset.max_zeros_batch([], 5) == []
    assert infoset.max_zeros_batch([[]], 5) == [0]
    assert infoset.max_zeros_batch([[7]], 1) == orc.max_zeros_batch(M, [[7]], 1)
    assert infoset.max_zeros_batch([[3, 3]], 1) == [49]
    assert infoset.max_zeros_batch([[5, 9, 5, 11, 12, 13, 14, 20, 30, 31, 40]], 1) == [49]
    assert infoset.max_zeros_batch([[0, 48]], 1) == orc.max_zeros_batch(M, [[0, 48]], 1)
    with pytest.raises(ValueError):
        infoset.max_zeros_batch([[0, 49]], 1)
    with pytest.raises(ValueError):
        infoset.max_zeros_batch([list(range(22))], 1)


def test_every_small_k_one_batch(M, infoset):
    rng = random.Random(303)
    sets = [sorted(rng.sample(range(N), k)) for k in range(2, 9) for _ in range(6)]
    assert infoset.max_zeros_batch(sets, 1) == orc.max_zeros_batch(M, sets, 1)


def test_matches_orbit_at_large_k(infoset, orbit):
    """Two independent enumerations agree where the oracle cannot run."""
    rng = random.Random(304)
    sets = rand_sets(rng, 40, 9, 13) + rand_sets(rng, 4, 14, 14)
    assert infoset.max_zeros_batch(sets, 1) == orbit.max_zeros_batch(sets, 1)


def test_large_k_threshold_decisions(infoset, orbit):
    rng = random.Random(305)
    sets = rand_sets(rng, 40, 10, 13)
    exact = orbit.max_zeros_batch(sets, 1)
    tds = [rng.randint(10, 30) for _ in sets]
    check_decisions(infoset.max_zeros_batch(sets, tds), exact, tds)


def test_auto_mixes_both_paths(M, orbit):
    """AUTO sends k >= 2 to information sets and k = 1 to the orbit walk,
    in one batch, with per-set thresholds."""
    from generalized_toric_gpu_search_b200 import _lib

    auto = oracle_for(M, _lib.TG_ENUM_AUTO)
    rng = random.Random(306)
    sets = rand_sets(rng, 120, 1, 13)
    exact = orbit.max_zeros_batch(sets, 1)
    assert auto.max_zeros_batch(sets, 1) == exact
    tds = [rng.randint(1, 35) for _ in sets]
    check_decisions(auto.max_zeros_batch(sets, tds), exact, tds)


@pytest.mark.parametrize("k", [15, 18, 21])
def test_agl2_invariance_at_large_k(infoset, k):
    """max_zeros is an AGL2(F7) invariant; the images pick other information
    sets, so agreement checks the bound logic at sizes nothing else reaches."""
    from generalized_toric_gpu_search_b200.tables import precompute_gl2_perms

    perms = precompute_gl2_perms()
    rng = random.Random(400 + k)
    base = [sorted(rng.sample(range(N), k)) for _ in range(3)]
    images = []
    for s in base:
        A = perms[rng.randrange(len(perms))]
        da, db = rng.randrange(7), rng.randrange(7)
        img = [int(A[i]) for i in s]
        images.append(sorted(((p // 7 + da) % 7) * 7 + (p % 7 + db) % 7 for p in img))
    a = infoset.max_zeros_batch(base, 1)
    assert a == infoset.max_zeros_batch(images, 1)
    # Singleton bound d <= 49 - k + 1, i.e. max_zeros >= k - 1
    assert all(z >= k - 1 for z in a)


def test_subcode_monotone_at_large_k(infoset):
    rng = random.Random(307)
    base = rand_sets(rng, 12, 12, 16)
    bigger = [sorted(s + [rng.choice([p for p in range(N) if p not in s])]) for s in base]
    a = infoset.max_zeros_batch(base, 1)
    b = infoset.max_zeros_batch(bigger, 1)
    assert all(y >= x for x, y in zip(a, b))


def test_any_evaluation_matrix():
    """Information sets need no toric structure: a random matrix with two equal
    rows and a zero row, against the oracle."""
    rng = np.random.default_rng(308)
    R = rng.integers(0, 8, size=(N, N)).astype(np.int32)
    R[5] = R[4]
    R[9] = 0
    o = oracle_for(R, INFOSET, variant=2)
    r = random.Random(309)
    sets = rand_sets(r, 60, 1, 7) + [[4, 5], [1, 9, 20], [4, 5, 30, 31]]
    assert o.max_zeros_batch(sets, 1) == orc.max_zeros_batch(R, sets, 1)


def test_counters_show_fewer_codewords(M, infoset):
    """At k = 14 the walk evaluates far fewer codewords than the projective
    count (8^14 - 1) / 7."""
    import torch

    from generalized_toric_gpu_search_b200.distance import DistanceRunner, LaunchConfig
    from generalized_toric_gpu_search_b200.distance import ToricContext

    rng = random.Random(310)
    sets = [sorted(rng.sample(range(N), 14)) for _ in range(4)]
    ctx = ToricContext(0, M)
    run = DistanceRunner(ctx, LaunchConfig(enumeration=INFOSET))
    flat = torch.tensor([i for s in sets for i in s], dtype=torch.int32, device="cuda:0")
    off = torch.tensor(np.cumsum([0] + [len(s) for s in sets]), dtype=torch.int64,
                       device="cuda:0")
    out = torch.empty(len(sets), dtype=torch.int32, device="cuda:0")
    p = run.params(len(sets), 14, 1)
    run.run(p, flat, off, out)
    tasks, codewords, ref = run.counters()
    assert out.tolist() == infoset.max_zeros_batch(sets, 1)
    assert 0 < codewords < len(sets) * (8 ** 14 - 1) // 7 // 20
    assert ref == pytest.approx(len(sets) * (8.0 ** 14 - 1))
