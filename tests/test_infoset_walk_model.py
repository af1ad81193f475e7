"""Host model of the block walk of the information-set kernel.

walk_level_kernel (csrc/infoset_kernel.cuh) enumerates, for each support of w
rows of an information set, the 7^(w-1) messages whose last support row has
coefficient 1 (the projective messages of that support):

  * a block is 49 codewords: digit 0 takes alpha^0..alpha^6 in each of 7
    sweeps, digit 1 steps alpha^0..alpha^6 between the sweeps and returns to
    alpha^0 with the move to the next block;
  * digits 2..w-2 follow a reflected base-7 Gray code over the block index b:
    block b starts with digit 2 + i at the base-7 digit o_i of b, reflected
    (6 - o_i) when the digits above it sum to an odd number, and the move
    into block m changes one digit by alpha^v + alpha^(v+1);
  * the move into block m is computed incrementally (m % 7 and the parity of
    m / 7) six times in seven, and by the general trailing-zero form
    otherwise.

This model applies those moves exactly as the kernel does, checks each block
against the closed-form start state, and checks that any split of a support
into tasks [b0, b0 + n) visits every projective message once.  It is the
coverage argument of the walk, independent of the GPU.
"""

from __future__ import annotations

import itertools
import random
from math import comb

import pytest

ALPHA = [1, 2, 4, 3, 6, 7, 5]  # alpha^e, alpha = x in GF(2)[x]/(x^3 + x + 1)


def block_digit_values(b: int, n_dig: int) -> list[int]:
    """Closed-form Gray values (exponents) of digits 2.. at the start of block b."""
    out, rest = [], b
    for _ in range(n_dig):
        o = rest % 7
        rest //= 7
        out.append(6 - o if rest & 1 else o)
    return out


def general_move(m: int) -> tuple[int, int]:
    """(digit index tz, step v): the move into block m changes digit 2 + tz
    between alpha^v and alpha^(v+1)."""
    tz = 0
    while m % 7 == 0:
        m //= 7
        tz += 1
    ot = m % 7
    return tz, (6 - ot if (m // 7) & 1 else ot - 1)


def walk_task(b0: int, n: int, n_dig: int) -> list[tuple[int, ...]]:
    """Messages (coefficients of digits 0, 1, 2.., GF(8) elements) of blocks
    [b0, b0 + n), in the kernel's order and with its state updates."""
    coef = [ALPHA[e] for e in block_digit_values(b0, n_dig)]
    m7, par = (b0 + 1) % 7, ((b0 + 1) // 7) & 1
    nxt = general_move(b0 + 1) if n > 1 else None
    seen = []
    for i in range(n):
        if i:
            tz, v = nxt
            coef[tz] ^= ALPHA[v] ^ ALPHA[(v + 1) % 7]
            assert coef == [ALPHA[e] for e in block_digit_values(b0 + i, n_dig)]
            m7 += 1
            if m7 == 7:
                m7, par = 0, par ^ 1
            if i + 1 < n:
                nxt = (0, 6 - m7 if par else m7 - 1) if m7 else general_move(b0 + i + 1)
        for s in range(7):  # digit 1 at alpha^s
            for v in range(7):  # digit 0 at alpha^v
                seen.append((ALPHA[v], ALPHA[s], *coef))
    return seen


@pytest.mark.parametrize("w", [3, 4, 5, 6])
def test_tasks_cover_every_projective_message(w):
    n_dig = w - 3
    bps = 7 ** n_dig
    rng = random.Random(w)
    for _ in range(5):
        cuts = sorted(rng.sample(range(1, bps), min(bps - 1, rng.randint(0, 6)))) if bps > 1 else []
        bounds = [0, *cuts, bps]
        seen = []
        for b0, b1 in zip(bounds, bounds[1:]):
            seen += walk_task(b0, b1 - b0, n_dig)
        assert len(seen) == 7 ** (w - 1)
        assert set(seen) == set(itertools.product(ALPHA, repeat=w - 1))


def test_incremental_moves_match_the_general_form():
    rng = random.Random(11)
    for _ in range(3000):
        b0, n = rng.randrange(7 ** 6), rng.randint(1, 343)
        m7, par = (b0 + 1) % 7, ((b0 + 1) // 7) & 1
        for i in range(1, n):
            m7 += 1
            if m7 == 7:
                m7, par = 0, par ^ 1
            if i + 1 < n and m7:
                assert (0, 6 - m7 if par else m7 - 1) == general_move(b0 + i + 1)


def test_digit1_return_is_alpha_squared():
    """Between blocks digit 1 goes alpha^6 -> alpha^0: a change of
    alpha^6 + 1 = alpha^2, applied on bit planes as (x1, x1 ^ x2, x0 ^ x2)."""
    assert ALPHA[6] ^ ALPHA[0] == ALPHA[2]

    def mul(a, b):
        r = 0
        for i in range(3):
            if (b >> i) & 1:
                r ^= a << i
        for i in (4, 3):
            if (r >> i) & 1:
                r ^= 0b1011 << (i - 3)
        return r

    for a in range(8):
        x0, x1, x2 = a & 1, (a >> 1) & 1, (a >> 2) & 1
        assert (x1 | (x1 ^ x2) << 1 | (x0 ^ x2) << 2) == mul(a, ALPHA[2])


def unrank_small_levels(k: int):
    """Units of levels 1-3 of one set, as levels123_kernel unranks them:
    rows, then pairs q < p, then triples q < p < t."""
    n1, n2, n3 = k, k * (k - 1) // 2, k * (k - 1) * (k - 2) // 6
    out = []
    for r in range(n1 + n2 + n3):
        if r < n1:
            out.append((r,))
            continue
        r -= n1
        t = -1
        if r >= n2:
            r -= n2
            t = 2
            while (t + 1) * t * (t - 1) // 6 <= r:
                t += 1
            r -= t * (t - 1) * (t - 2) // 6
        p = 1
        while (p + 1) * p // 2 <= r:
            p += 1
        q = r - p * (p - 1) // 2
        out.append((q, p) if t < 0 else (q, p, t))
    return out


@pytest.mark.parametrize("k", [1, 2, 3, 7, 14, 21])
def test_levels123_unranking_covers_every_support(k):
    got = unrank_small_levels(k)
    want = [c for w in (1, 2, 3) for c in itertools.combinations(range(k), w)]
    assert sorted(got) == sorted(want) and len(got) == len(want)


def unrank_support(k: int, w: int, rank: int) -> tuple[int, ...]:
    """Rows of the support of rank `rank` at level w, unranked as
    is_walk_range does: from row k - 1 down, take row pos when the remaining
    rank is at least C(pos, rem)."""
    rows, rem = [], w
    for pos in range(k - 1, -1, -1):
        if rem == 0:
            break
        b = comb(pos, rem)
        if rank < b:
            continue
        rank -= b
        rem -= 1
        rows.append(pos)
    assert rem == 0
    return tuple(sorted(rows))


def part_supports(k: int, w: int, part: int) -> tuple[int, int]:
    """(count, first rank) of a toric code's supports in part `part` of level
    w, as is_part_supports gives them."""
    if part == 1:
        return comb(k - 1, w - 1), comb(k - 1, w)
    return comb(k - 1, w), 0


@pytest.mark.parametrize("k", [4, 5, 9, 14])
def test_level_parts_split_supports_by_the_last_row(k):
    """Part 1 of level w holds exactly the supports with row k - 1, part 2
    the others; together every w-subset of the rows once."""
    for w in range(4, k + 1):
        seen = []
        for part in (1, 2):
            n_sup, s_off = part_supports(k, w, part)
            sup = [unrank_support(k, w, s_off + s) for s in range(n_sup)]
            assert all(((k - 1) in x) == (part == 1) for x in sup)
            seen += sup
        assert sorted(seen) == list(itertools.combinations(range(k), w))

