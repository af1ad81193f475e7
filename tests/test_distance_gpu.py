"""Parity of the B200 max_zeros kernels with the oracle and the reference.

Bit-exact contract (the reference's, kernel_cuda_bp.py:227-235): a passing set
returns exactly max_zeros; a failing set returns a value > 49 - td.
"""

from __future__ import annotations

import random

import numpy as np
import pytest

from oracle import oracle as orc

pytestmark = pytest.mark.gpu

N = 49


def rand_sets(rng, n, kmin, kmax):
    return [sorted(rng.sample(range(N), rng.randint(kmin, kmax))) for _ in range(n)]


def check_decisions(got, exact, tds):
    for g, e, td in zip(got, exact, tds):
        tmax = N - td
        if e <= tmax:
            assert g == e
        else:
            assert g > tmax


def test_known_answers(gpu_oracle, golden):
    sets = [k["set"] for k in golden["max_zeros_kats"]]
    want = [k["max_zeros"] for k in golden["max_zeros_kats"]]
    assert gpu_oracle.max_zeros_batch(sets, 1) == want
    for s, w in zip(sets, want):
        assert gpu_oracle.max_zeros(s, 1) == w


def test_reference_smoke_tests(gpu_oracle):
    # kernel backup.py:180-245
    assert gpu_oracle.max_zeros([0], 49) == 0
    assert gpu_oracle.max_zeros([0, 1, 7], 1) == 7
    assert gpu_oracle.max_zeros([0, 1, 7], 49) > 0          # early abort reports a fail
    assert gpu_oracle.max_zeros([0, 1, 7], 42) == 7         # loose target: exact
    assert gpu_oracle.min_distance([0, 8, 18, 23, 30, 39, 43]) == 34   # parabola conic
    assert gpu_oracle.min_distance([1, 6, 7, 16, 19, 37, 40, 42]) == 24  # circle conic


@pytest.mark.parametrize("enumeration,variant", [(0, 0), (1, 1), (2, 1), (1, 2), (2, 2)])
@pytest.mark.parametrize("tail_rows", [0, 2, 3, 5])
def test_random_mixed_k_exact(M, enumeration, variant, tail_rows):
    from generalized_toric_gpu_search_b200.distance import DistanceOracleCUDABP, LaunchConfig

    rng = random.Random(100 + 7 * enumeration + variant + 31 * tail_rows)
    sets = rand_sets(rng, 60, 1, 7)
    want = orc.max_zeros_batch(M, sets, 1)
    o = DistanceOracleCUDABP(0, M, LaunchConfig(tail_rows=tail_rows, enumeration=enumeration,
                                                variant=variant))
    assert o.max_zeros_batch(sets, 1) == want


def test_config_c1_plain_k8(gpu_oracle, M):
    """64 seeded sets of k = 8 (the CPU-runnable configuration), td = 1."""
    rng = np.random.default_rng(1)
    sets = [sorted(rng.choice(N, 8, replace=False).tolist()) for _ in range(64)]
    want = orc.max_zeros_batch(M, sets, 1)
    assert gpu_oracle.max_zeros_batch(sets, 1) == want


def test_thresholds_decisions(gpu_oracle, M):
    rng = random.Random(7)
    sets = rand_sets(rng, 120, 2, 7)
    exact = orc.max_zeros_batch(M, sets, 1)
    tds = [rng.randint(1, 49) for _ in sets]
    got = gpu_oracle.max_zeros_batch(sets, tds)
    check_decisions(got, exact, tds)
    for td in (20, 30, 40, 45):
        got = gpu_oracle.max_zeros_batch(sets, td)
        check_decisions(got, exact, [td] * len(sets))


def test_edge_cases(gpu_oracle, M):
    assert gpu_oracle.max_zeros_batch([], 5) == []
    assert gpu_oracle.max_zeros([], 5) == 0
    assert gpu_oracle.max_zeros_batch([[]], 5) == [0]
    assert gpu_oracle.max_zeros_batch([[3, 3]], 1) == [49]        # dependent rows
    assert gpu_oracle.max_zeros_batch([[5, 9, 5, 11]], 1) == [49]
    assert gpu_oracle.max_zeros_batch([[0, 48]], 1) == orc.max_zeros_batch(M, [[0, 48]], 1)
    with pytest.raises(ValueError):
        gpu_oracle.max_zeros_batch([list(range(22))], 1)
    with pytest.raises(ValueError):
        gpu_oracle.max_zeros(list(range(22)), 1)
    with pytest.raises(ValueError):
        gpu_oracle.max_zeros_batch([list(range(50))], 1, sample_count=10)
    with pytest.raises(ValueError):
        gpu_oracle.max_zeros_batch([[0, 49]], 1)
    with pytest.raises(ValueError):
        gpu_oracle.max_zeros_batch([[-1, 3]], 1)


@pytest.mark.parametrize("k", [3, 6, 12, 21, 22, 30, 49])
def test_sampled_bit_exact(gpu_oracle, M, k):
    rng = random.Random(1000 + k)
    sets = [sorted(rng.sample(range(N), k)) for _ in range(12)]
    for seed in (0, 12345, 2**63 + 17):
        want = orc.max_zeros_batch(M, sets, 1, sample_count=3000, sample_seed=seed)
        got = gpu_oracle.max_zeros_batch(sets, 1, sample_count=3000, sample_seed=seed)
        assert got == want


def test_sampled_threshold_decisions(gpu_oracle, M):
    rng = random.Random(5)
    sets = [sorted(rng.sample(range(N), 9)) for _ in range(40)]
    full = orc.max_zeros_batch(M, sets, 1, sample_count=5000, sample_seed=99)
    got = gpu_oracle.max_zeros_batch(sets, 30, sample_count=5000, sample_seed=99)
    check_decisions(got, full, [30] * len(sets))


def test_invariance_under_agl2(gpu_oracle):
    """Size-independent property: max_zeros is an AGL2(F7) invariant."""
    from generalized_toric_gpu_search_b200.tables import precompute_gl2_perms

    perms = precompute_gl2_perms()
    rng = random.Random(11)
    base = rand_sets(rng, 24, 9, 12)
    images = []
    for s in base:
        A = perms[rng.randrange(len(perms))]
        da, db = rng.randrange(7), rng.randrange(7)
        img = [int(A[i]) for i in s]
        images.append(sorted(((p // 7 + da) % 7) * 7 + (p % 7 + db) % 7 for p in img))
    assert gpu_oracle.max_zeros_batch(base, 1) == gpu_oracle.max_zeros_batch(images, 1)


def test_subcode_monotone(gpu_oracle):
    """Adding a row can only add codewords: max_zeros never decreases."""
    rng = random.Random(13)
    base = rand_sets(rng, 30, 8, 11)
    bigger = []
    for s in base:
        extra = rng.choice([p for p in range(N) if p not in s])
        bigger.append(sorted(s + [extra]))
    a = gpu_oracle.max_zeros_batch(base, 1)
    b = gpu_oracle.max_zeros_batch(bigger, 1)
    assert all(y >= x for x, y in zip(a, b))


def test_orbit_matches_projective_at_k12(M):
    """Two independent enumerations agree at sizes the oracle cannot run."""
    from generalized_toric_gpu_search_b200.distance import DistanceOracleCUDABP, LaunchConfig

    rng = random.Random(17)
    sets = rand_sets(rng, 6, 11, 12)
    orbit = DistanceOracleCUDABP(0, M, LaunchConfig(enumeration=2, variant=1))
    proj = DistanceOracleCUDABP(0, M, LaunchConfig(enumeration=1, variant=2))
    assert orbit.max_zeros_batch(sets, 1) == proj.max_zeros_batch(sets, 1)
