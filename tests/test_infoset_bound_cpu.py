"""The lower bounds the information-set walk stops on, checked by brute force
on small toric codes (every codeword enumerated on the CPU).

With E an information set of a k-row toric code, the translates E + t (the
torus translations (x, y) -> (lambda x, mu y)) are information sets too, and
the walk on E meets, up to a translation, every codeword that weighs w on
some translate.  plan_level_kernel stops a code on these bounds for the
codewords it has not met:

  * after levels 1..w-1: weight >= ceil(49 w / k);
  * after levels 1..w-1 and part 1 of level w (the supports holding the row of
    pivot column e): weight >= ceil(49 w / (k - 1)).

A codeword c is met by part 1 of level w when some translate of c weighs w
on E and is nonzero at e.  This test enumerates every codeword of random
toric codes with k = 3..6, every information-set column e and every level,
and checks both bounds against the lightest codeword not met.  It is the
coverage argument of the two-part levels, independent of the GPU.
"""

from __future__ import annotations

import itertools

import numpy as np
import pytest

from generalized_toric_gpu_search_b200.tables import MUL_TABLE, build_eval_matrix, gf8_mul

N = 49


def all_codewords(G: np.ndarray) -> np.ndarray:
    """Every codeword u G of the k x 49 GF(8) generator G, as (8^k, 49)."""
    cw = np.zeros((1, N), dtype=np.uint8)
    for row in G:
        mult = MUL_TABLE[np.arange(8)][:, row]  # (8, 49): a * row for a in GF(8)
        cw = (cw[:, None, :] ^ mult[None, :, :]).reshape(-1, N)
    return cw


def translations() -> np.ndarray:
    """(49, 49): row t is the column permutation of one torus translation;
    the translate of c is c[perm]."""
    col = {(1 + j // 7, 1 + j % 7): j for j in range(N)}
    out = []
    for lam in range(1, 8):
        for mu in range(1, 8):
            out.append([col[(gf8_mul(lam, 1 + j // 7), gf8_mul(mu, 1 + j % 7))] for j in range(N)])
    return np.asarray(out, dtype=np.int64)


def information_set(support: np.ndarray, k: int, rng) -> list[int]:
    """k columns on which no nonzero codeword vanishes (so u G -> c|E is a
    bijection)."""
    nz = support[1:]
    for _ in range(10_000):
        E = sorted(rng.choice(N, k, replace=False).tolist())
        if nz[:, E].any(axis=1).all():
            return E
    raise AssertionError("no information set found")


def ceil_div(a: int, b: int) -> int:
    return -(-a // b)


@pytest.mark.parametrize("k,seed", [(3, 1), (4, 2), (4, 3), (5, 4), (5, 5), (6, 6)])
def test_level_and_part_bounds_hold(k, seed):
    rng = np.random.default_rng(seed)
    M = build_eval_matrix()
    P = sorted(rng.choice(N, k, replace=False).tolist())
    cw = all_codewords(M[P].astype(np.uint8))
    S = cw != 0
    wt = S.sum(axis=1)
    assert (wt[1:] > 0).all()
    E = information_set(S, k, rng)
    perm = translations()
    # weight on E of every translate of every codeword: (8^k, 49)
    onE = np.stack([S[:, perm[t]][:, E].sum(axis=1) for t in range(N)], axis=1)
    nz = np.arange(len(cw)) > 0
    checked = parts = 0
    for w in range(1, k + 1):
        met_before = (onE < w).any(axis=1)
        rest = nz & ~met_before
        if rest.any():
            assert wt[rest].min() >= ceil_div(N * w, k)
            checked += 1
        if k < 2:
            continue
        for e in E:
            # translate t is nonzero at e exactly when c is nonzero at perm[t][e]
            at_e = np.stack([S[:, perm[t][e]] for t in range(N)], axis=1)
            met = met_before | ((onE == w) & at_e).any(axis=1)
            rest = nz & ~met
            if rest.any():
                assert wt[rest].min() >= ceil_div(N * w, k - 1), (P, E, e, w)
                parts += 1
    assert checked > 0 and parts > 0


def test_part_bound_can_exceed_the_level_bound():
    """The part-1 bound is the one that lets a code stop half-way through a
    level: at k = 13 it reaches 21 after part 1 of level 5, where levels 1..4
    give 19 and level 5 whole gives 23."""
    assert ceil_div(N * 5, 13) == 19
    assert ceil_div(N * 5, 12) == 21
    assert ceil_div(N * 6, 13) == 23
    for k, w in itertools.product(range(4, 22), range(4, 12)):
        if w < k:
            assert ceil_div(N * w, k) <= ceil_div(N * w, k - 1) <= ceil_div(N * (w + 1), k)
