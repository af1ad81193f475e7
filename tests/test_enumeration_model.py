"""Host model of the message enumeration the distance kernels walk.

The prep kernel orders the rows (leading head rows in general position),
splits them into H head rows (normalised message patterns) and R tail rows
(walked completely inside one task), and emits the patterns:
  zero head; one nonzero head coefficient = 1; two = (1, 1); three or more
  with the first three (1, 1, c), c = 1 unless the three exponent points are
  collinear (then c in 1..7), the rest free.        (orbit enumeration)
  first nonzero head coefficient = 1, the rest free. (projective enumeration)
This model restates that plan in Python and checks on small codes that the
largest zero count over the enumerated messages equals the exhaustive
max_zeros of the oracle -- the correctness argument of the torus-orbit
reduction, independent of the GPU.
"""

from __future__ import annotations

import itertools
import random

import numpy as np
import pytest

from oracle import oracle as orc


def collinear(p, q, r):
    ua, ub = q // 7 - p // 7, q % 7 - p % 7
    va, vb = r // 7 - p // 7, r % 7 - p % 7
    return (ua * vb - ub * va) % 7 == 0


def row_order(S, H, orbit):
    k = len(S)
    used, order = set(), []
    if orbit:
        for _ in range(H):
            best, best_cost = None, None
            for cand in range(k):
                if cand in used:
                    continue
                cost = sum(collinear(S[order[x]], S[order[y]], S[cand])
                           for x in range(len(order)) for y in range(x + 1, len(order)))
                if best_cost is None or cost < best_cost:
                    best, best_cost = cand, cost
            order.append(best)
            used.add(best)
    order += [c for c in range(k) if c not in used]
    return [S[i] for i in order]


def head_vectors(rows, H, orbit):
    """Yields the head coefficient vectors of every task."""
    yield [0] * H
    if orbit:
        for i0 in range(H):
            v = [0] * H
            v[i0] = 1
            yield v
        for i0, i1 in itertools.combinations(range(H), 2):
            v = [0] * H
            v[i0] = v[i1] = 1
            yield v
        for i0, i1, i2 in itertools.combinations(range(H), 3):
            cs = range(1, 8) if collinear(rows[i0], rows[i1], rows[i2]) else [1]
            for c in cs:
                for free in itertools.product(range(8), repeat=H - 1 - i2):
                    v = [0] * H
                    v[i0] = v[i1] = 1
                    v[i2] = c
                    v[i2 + 1:] = list(free)
                    yield v
    else:
        for i0 in range(H):
            for free in itertools.product(range(8), repeat=H - 1 - i0):
                v = [0] * H
                v[i0] = 1
                v[i0 + 1:] = list(free)
                yield v


def model_max_zeros(S, M, R, orbit):
    mul = orc.mul_table()
    k = len(S)
    R = min(R, k)
    H = k - R
    rows = row_order(list(S), H, orbit)
    G = [M[r].astype(np.int64) for r in rows]
    best, tasks = 0, 0
    tails = list(itertools.product(range(8), repeat=R))
    for head in head_vectors(rows, H, orbit):
        tasks += 1
        base = np.zeros(49, dtype=np.int64)
        for c, g in zip(head, G[:H]):
            if c:
                base ^= mul[c][g]
        for tail in tails:
            if not any(head) and not any(tail):
                continue  # the zero message
            v = base.copy()
            for c, g in zip(tail, G[H:]):
                if c:
                    v ^= mul[c][g]
            best = max(best, int((v == 0).sum()))
    return best, tasks


@pytest.mark.parametrize("orbit", [True, False])
@pytest.mark.parametrize("R", [2, 3])
def test_enumeration_covers_every_orbit(M, orbit, R):
    rng = random.Random(41 + R + 10 * orbit)
    for _ in range(5):
        k = rng.randint(2, 6)
        S = rng.sample(range(49), k)
        got, _ = model_max_zeros(S, M, R, orbit)
        assert got == orc.max_zeros_batch(M, [S], 1)[0], S


def test_collinear_head_rows(M):
    # all points on the line a = 0: every head triple is collinear
    S = [0, 1, 2, 3, 4, 5]
    got, _ = model_max_zeros(S, M, 2, True)
    assert got == orc.max_zeros_batch(M, [S], 1)[0]


def test_orbit_uses_fewer_tasks(M):
    S = [0, 8, 18, 23, 30, 39, 43]
    _, t_orbit = model_max_zeros(S, M, 3, True)
    _, t_proj = model_max_zeros(S, M, 3, False)
    assert t_orbit < t_proj
