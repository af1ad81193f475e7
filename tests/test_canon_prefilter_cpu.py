"""The first-row prefilter of the canonical form (canon_mask_warp_min), as a
host model against brute force.

The canonical mask of S is the smallest mask among the translates, anchored
at their points, of the images A S over GL2(F7).  A candidate's order is
decided first by its top row.  The image of (x, y) under A = (a b; c d)
lies in row a x + b y, so the row occupancy of A S, and with it the smallest
top row its anchored translates can reach, depends on A's first row alone;
the table lists the matrices by (a, b, c, d), 42 per first row.  The kernel
keeps only the first rows that reach the overall smallest top row.  This test
checks, on random sets of every size, that the minimum over those first rows
equals the minimum over all 2016 matrices.  The last test checks the host
assembly of compute()'s packed keys.
"""

from __future__ import annotations

import numpy as np
import pytest

from generalized_toric_gpu_search_b200.tables import precompute_gl2_perms

N = 49
PERMS = precompute_gl2_perms()


def translates(img_idx: np.ndarray) -> list[int]:
    """Masks of the image translated by -q for each of its points q."""
    xs, ys = img_idx // 7, img_idx % 7
    out = []
    for qa, qb in zip(xs.tolist(), ys.tolist()):
        m = 0
        for x, y in zip(xs.tolist(), ys.tolist()):
            m |= 1 << (((x - qa) % 7) * 7 + (y - qb) % 7)
        out.append(m)
    return out


def canonical_brute(S: list[int], mats) -> int:
    return min(min(translates(PERMS[a][S])) for a in mats)


def min_top_row(rows: set[int]) -> int:
    return min(max((r - qa) % 7 for r in rows) for qa in rows)


@pytest.mark.parametrize("size", [1, 2, 3, 5, 8, 13, 20, 30, 45])
def test_first_row_prefilter_keeps_the_minimum(size):
    rng = np.random.default_rng(100 + size)
    for _ in range(6):
        S = sorted(rng.choice(N, size, replace=False).tolist())
        tops = []
        for g in range(48):
            rows = set((PERMS[g * 42][S] // 7).tolist())
            # every matrix of the group has the same image rows
            assert all(set((PERMS[g * 42 + j][S] // 7).tolist()) == rows for j in (1, 20, 41))
            tops.append(min_top_row(rows))
        tstar = min(tops)
        kept = [g * 42 + j for g in range(48) if tops[g] == tstar for j in range(42)]
        assert canonical_brute(S, kept) == canonical_brute(S, range(2016))
        assert (canonical_brute(S, kept).bit_length() - 1) // 7 == tstar


def test_keys_from_words_matches_the_reference_formula():
    """compute()'s key assembly: Python ints lo + hi * 2**64
    (kernel_canon.py:174-176), whether or not a row has a high word."""
    from generalized_toric_gpu_search_b200.canonical import keys_from_words

    rng = np.random.default_rng(3)
    lo = rng.integers(0, 2**63, 5000, dtype=np.uint64) * np.uint64(2) + np.uint64(1)
    for hi in (np.zeros(5000, np.uint64), rng.integers(0, 2**32, 5000, dtype=np.uint64),
               np.where(rng.random(5000) < 0.1, np.uint64(7), np.uint64(0))):
        got = keys_from_words(lo, hi)
        want = lo.astype(object) + hi.astype(object) * (1 << 64)
        assert got.dtype == object and len(got) == 5000
        assert all(type(g) is int and g == w for g, w in zip(got, want))
    assert len(keys_from_words(np.zeros(0, np.uint64), np.zeros(0, np.uint64))) == 0
