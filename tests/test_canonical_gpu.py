"""Parity of the B200 canonical-form kernel and dedup with the oracle."""

from __future__ import annotations

import random

import numpy as np
import pytest

from oracle import oracle as orc

pytestmark = pytest.mark.gpu

N = 49


def test_golden_keys(canon_oracle, golden):
    by_k = {}
    for rec in golden["canonical_keys"]:
        by_k.setdefault(len(rec["set"]), []).append(rec)
    for k, recs in by_k.items():
        sets = np.array([r["set"] for r in recs], dtype=np.int32)
        got = canon_oracle.compute(sets)
        assert [int(x) for x in got] == [r["key"] for r in recs]


@pytest.mark.parametrize("k", [11, 12, 13, 14, 15, 16])
def test_keys_k11_to_16_vs_oracle(canon_oracle, k):
    rng = random.Random(k)
    sets = np.array([sorted(rng.sample(range(N), k)) for _ in range(40)], dtype=np.int32)
    want = orc.canonical_keys(sets)
    got = canon_oracle.compute(sets)
    assert [int(x) for x in got] == want


def test_masks_any_k_vs_oracle(canon_oracle):
    rng = random.Random(3)
    masks = []
    for _ in range(300):
        k = rng.randint(1, 30)
        m = 0
        for p in rng.sample(range(N), k):
            m |= 1 << p
        masks.append(m)
    masks = np.array(masks, dtype=np.uint64)
    want = orc.canonical_masks(masks)
    got = canon_oracle.compute_masks(masks)
    assert np.array_equal(got, want)


def test_edge_sets(canon_oracle):
    full = np.arange(N, dtype=np.int32)[None, :]
    assert int(canon_oracle.compute_masks(full)[0]) == (1 << N) - 1
    one = np.array([[37]], dtype=np.int32)
    assert [int(x) for x in canon_oracle.compute(one)] == [0]
    assert canon_oracle.compute(np.zeros((0, 5), dtype=np.int32)).shape == (0,)
    empty_rows = canon_oracle.compute(np.zeros((3, 0), dtype=np.int32))
    assert [int(x) for x in empty_rows] == [(1 << 128) - 1] * 3
    with pytest.raises(ValueError):
        canon_oracle.compute(np.array([[1, 1, 2]], dtype=np.int32))
    with pytest.raises(ValueError):
        canon_oracle.compute(np.zeros((1, 17), dtype=np.int32))


def test_invariance_and_orbit_counts(canon_oracle):
    from generalized_toric_gpu_search_b200.tables import precompute_gl2_perms

    perms = precompute_gl2_perms()
    rng = random.Random(9)
    base, moved = [], []
    for _ in range(200):
        k = rng.randint(2, 25)
        s = rng.sample(range(N), k)
        A = perms[rng.randrange(len(perms))]
        da, db = rng.randrange(7), rng.randrange(7)
        t = [(int(A[p]) // 7 + da) % 7 * 7 + (int(A[p]) % 7 + db) % 7 for p in s]
        base.append(sum(1 << p for p in s))
        moved.append(sum(1 << p for p in t))
    a = canon_oracle.compute_masks(np.array(base, dtype=np.uint64))
    b = canon_oracle.compute_masks(np.array(moved, dtype=np.uint64))
    assert np.array_equal(a, b)
    # orbit counts of 2- and 3-subsets (1 and 3 classes)
    from itertools import combinations

    for k, classes in ((2, 1), (3, 3)):
        sets = np.array(list(combinations(range(N), k)), dtype=np.int32)
        assert len(set(canon_oracle.compute_masks(sets).tolist())) == classes


def test_dedup_first_occurrence(canon_oracle):
    from generalized_toric_gpu_search_b200.canonical import CanonicalDedup

    rng = np.random.default_rng(4)
    keys = rng.integers(0, 50, size=1000).astype(np.uint64)
    d = CanonicalDedup(0, capacity=4096)
    is_new = d.insert(keys)
    seen, want = set(), []
    for k in keys.tolist():
        want.append(k != 0 and k not in seen)  # 0 is not a key: never new
        seen.add(k)
    assert 0 in keys.tolist()
    assert is_new.tolist() == want
    again = d.insert(np.array([3, 60, 60, 1000], dtype=np.uint64))
    assert again.tolist() == [3 not in seen, True, False, True]
