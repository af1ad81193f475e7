"""Witness codewords (tg_max_zeros_witness) checked on the host by the oracle.

Every set's witness must be a codeword of its own code -- the oracle solves
m M[S] = c over GF(8) and re-evaluates m M[S] -- with exactly the reported
number of zeros.  For a passing set that proves the reported max_zeros is
reached; for a failing set it proves the failure decision, independently of
the walk that found it.  The workloads are the early-exit configuration
(2,000 seeded sets of k = 15 at the k = 15 best-known distance) and the full
batched mixed-k workload (10,000 seeded sets, k = 6..14), whose failures and
values are otherwise out of the reference's reach at these sizes.
"""

from __future__ import annotations

import random

import numpy as np
import pytest

from oracle import oracle as orc

pytestmark = pytest.mark.gpu

N = 49


def check_witnesses(M, sets, values, witnesses):
    for s, v, w in zip(sets, values, witnesses):
        if len(s) == 0:
            assert v == 0 and not w.any()
            continue
        zeros, msg = orc.codeword_message(M, s, w)
        assert zeros == v, (s, v, zeros)
        assert any(msg), s


def test_witness_small_k_matches_oracle(gpu_oracle, M):
    rng = random.Random(61)
    sets = [sorted(rng.sample(range(N), rng.randint(1, 8))) for _ in range(300)]
    values, wit = gpu_oracle.max_zeros_batch_witness(sets, 1)
    assert values == orc.max_zeros_batch(M, sets, 1)
    check_witnesses(M, sets, values, wit)


def test_witness_thresholds(gpu_oracle, M):
    rng = random.Random(62)
    sets = [sorted(rng.sample(range(N), rng.randint(4, 11))) for _ in range(400)]
    tds = [rng.randint(18, 40) for _ in sets]
    exact = gpu_oracle.max_zeros_batch(sets, 1)
    values, wit = gpu_oracle.max_zeros_batch_witness(sets, tds)
    for e, v, td in zip(exact, values, tds):
        tmax = N - td
        assert (v > tmax) == (e > tmax)
        if e <= tmax:
            assert v == e
        else:
            assert tmax < v <= e
    check_witnesses(M, sets, values, wit)


def test_witness_early_exit_k15(gpu_oracle, M):
    """The early-exit configuration: 2,000 seeded sets with |P| = 15 at the
    k = 15 best-known distance 24.  Every failure is proven by its witness."""
    from bench import BASE_SEED, FALLBACK_BEST_D

    rng = np.random.default_rng(BASE_SEED + 5)
    sets = [sorted(rng.choice(N, 15, replace=False).tolist()) for _ in range(2000)]
    td = FALLBACK_BEST_D[15]
    plain = gpu_oracle.max_zeros_batch(sets, td)
    values, wit = gpu_oracle.max_zeros_batch_witness(sets, td)
    tmax = N - td
    assert [v > tmax for v in values] == [p > tmax for p in plain]
    assert sum(v > tmax for v in values) > 1900
    check_witnesses(M, sets, values, wit)
    for p, v in zip(plain, values):
        if p <= tmax:
            assert v == p


def test_witness_batched_mixed_k_workload(gpu_oracle, M):
    """Every value of the 10,000-set batched workload (td = 1) is reached by
    a codeword the oracle verifies."""
    from bench import make_workload

    sets = make_workload(0)
    plain = gpu_oracle.max_zeros_batch(sets, 1)
    values, wit = gpu_oracle.max_zeros_batch_witness(sets, 1)
    assert values == plain
    check_witnesses(M, sets, values, wit)


def test_witness_non_toric_matrix_with_dependent_rows():
    from generalized_toric_gpu_search_b200.distance import DistanceOracleCUDABP

    rng = np.random.default_rng(63)
    M = rng.integers(0, 8, size=(N, N)).astype(np.int32)
    M[10] = M[3]
    M[11] = 0
    o = DistanceOracleCUDABP(0, M, autotune=False)
    r = random.Random(64)
    sets = [sorted(r.sample(range(N), r.randint(1, 9))) for _ in range(120)]
    sets += [[3, 10, 20], [11, 4], [3, 5, 10, 30, 31]]
    values, wit = o.max_zeros_batch_witness(sets, 1)
    assert values == orc.max_zeros_batch(M, sets, 1)
    for s, v, w in zip(sets, values, wit):
        if v == N:
            assert not w.any()  # dependent rows: the zero codeword
            continue
        zeros, msg = orc.codeword_message(M, s, w)
        assert zeros == v and any(msg)
