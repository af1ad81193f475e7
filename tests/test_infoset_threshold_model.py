"""Host model of the threshold test of the information-set walk
(is_walk_blocks, TG_IS_SWEEP1 / TG_IS_SWEEP1F / TG_IS_SWEEP2 and
is_block_fix in csrc/infoset_kernel.cuh).

Per support the walk works on the 32 low columns in the domain W = P h,
h = g^-1 column-wise (g the digit-0 row): the codeword P + alpha^v g is zero
at column j exactly when W_j = alpha^v (g_j != 0) or P_j = 0 (g_j = 0).  So a
sweep's seven zero counts are seven selections of W plus the zeros of P on
g's zero columns (Pz = P & gz), and digit 1's moves enter W as d h and Pz as
d & gz.  With the high columns weighing at least hb, a sweep can hold a
codeword lighter than wmin only if some count passes thr = 32 + hb - wmin;
the paired form bounds two codewords by one count of two disjoint
selections; the flagged forms count the flagged sweeps after the block by
stepping back through digit 1's moves.

This test restates those steps on Python integers (bit planes of 32
columns), with the kernel's bit-sliced product and inverse, and checks them
against per-column GF(8) arithmetic: the counts, the bounds (no sweep with a
lighter codeword is left unflagged), the step back, and that the on-the-spot
and flagged procedures find the same minimum as a direct scan of the block.
"""

from __future__ import annotations

import random

import pytest

LOW = 32
M32 = (1 << LOW) - 1
ALPHA = [1, 2, 4, 3, 6, 7, 5]  # alpha^e, alpha = x in GF(2)[x]/(x^3 + x + 1)


def gf_mul(a: int, b: int) -> int:
    r = 0
    for i in range(3):
        if (b >> i) & 1:
            r ^= a << i
    for i in (4, 3):
        if (r >> i) & 1:
            r ^= 0b1011 << (i - 3)
    return r


def gf_inv(a: int) -> int:
    return 0 if a == 0 else next(x for x in range(1, 8) if gf_mul(a, x) == 1)


def planes(vals: list[int]) -> tuple[int, int, int]:
    return tuple(sum(((v >> b) & 1) << j for j, v in enumerate(vals)) for b in range(3))


def values(p: tuple[int, int, int]) -> list[int]:
    return [((p[0] >> j) & 1) | (((p[1] >> j) & 1) << 1) | (((p[2] >> j) & 1) << 2)
            for j in range(LOW)]


def pl3_mul(a, b):
    """The kernel's bit-sliced column-wise product."""
    t0 = a[0] & b[0]
    t1 = (a[0] & b[1]) ^ (a[1] & b[0])
    t2 = (a[0] & b[2]) ^ (a[1] & b[1]) ^ (a[2] & b[0])
    t3 = (a[1] & b[2]) ^ (a[2] & b[1])
    t4 = a[2] & b[2]
    return (t0 ^ t3, t1 ^ t3 ^ t4, t2 ^ t4)


def pl3_inv(a):
    """The kernel's column-wise inverse a^6 = a^2 a^4 (0 stays 0)."""
    s2 = (a[0], a[2], a[1] ^ a[2])
    s4 = (s2[0], s2[2], s2[1] ^ s2[2])
    return pl3_mul(s2, s4)


def pl3_xor(a, b):
    return (a[0] ^ b[0], a[1] ^ b[1], a[2] ^ b[2])


def pl3_and(a, m):
    return (a[0] & m, a[1] & m, a[2] & m)


def pl3_alpha(a):
    return (a[2], a[0] ^ a[2], a[1])


def sel(W, v: int) -> int:
    """Columns where W equals the GF(8) value v."""
    m = M32
    for b in range(3):
        m &= W[b] if (v >> b) & 1 else ~W[b] & M32
    return m


def nz(p) -> int:
    return bin((p[0] | p[1] | p[2]) & M32).count("1")


def random_row(rng: random.Random, zero_frac: float) -> list[int]:
    return [0 if rng.random() < zero_frac else rng.randrange(1, 8) for _ in range(LOW)]


def block_state(rng: random.Random, zero_frac: float = 0.15):
    """A block: g (digit 0), r1 (digit 1), P (the other digits' sum) on the
    low columns."""
    g = random_row(rng, zero_frac)
    r1 = random_row(rng, 0.1)
    P = random_row(rng, 0.1)
    return g, r1, P


def digit1_moves(r1p, h, gz):
    """Digit 1's six steps (alpha^i + alpha^(i+1)) r1 in both domains: one
    product with h, then a multiplication by alpha per step."""
    d0 = pl3_xor(r1p, pl3_alpha(r1p))  # (1 + alpha) r1
    e, zq = pl3_mul(d0, h), pl3_and(d0, gz)
    out = []
    for _ in range(6):
        out.append((e, zq))
        e, zq = pl3_alpha(e), pl3_alpha(zq)
    return out


def sweeps(g, r1, P):
    """The seven sweeps of one block, as (W, Pz) states and the true
    low-column zero counts of their 7 codewords."""
    gp, r1p, Pp = planes(g), planes(r1), planes(P)
    h = pl3_inv(gp)
    gz = ~(gp[0] | gp[1] | gp[2]) & M32
    mv = digit1_moves(r1p, h, gz)
    P0 = pl3_xor(Pp, r1p)  # digit 1 starts the block at alpha^0
    W, Pz = pl3_mul(P0, h), pl3_and(P0, gz)
    states, truth = [], []
    for s in range(7):
        cur = [p ^ gf_mul(ALPHA[s], r) for p, r in zip(P, r1)]  # digit 1 at alpha^s
        truth.append([sum(1 for p, x in zip(cur, g) if p == gf_mul(ALPHA[v], x))
                      for v in range(7)])
        states.append((W, Pz))
        if s < 6:
            W, Pz = pl3_xor(W, mv[s][0]), pl3_xor(Pz, mv[s][1])
    return states, truth, mv, bin(gz).count("1")


@pytest.mark.parametrize("seed", range(40))
def test_w_domain_counts_equal_the_codewords_zeros(seed):
    rng = random.Random(seed)
    g, r1, P = block_state(rng, zero_frac=[0.0, 0.1, 0.3, 0.6][seed % 4])
    gp = planes(g)
    assert values(pl3_mul(gp, pl3_inv(gp))) == [1 if x else 0 for x in g]
    assert values(pl3_mul(planes(P), gp)) == [gf_mul(p, x) for p, x in zip(P, g)]
    assert values(pl3_inv(gp)) == [gf_inv(x) for x in g]
    states, truth, _, ngz = sweeps(g, r1, P)
    for (W, Pz), want in zip(states, truth):
        z = [bin(sel(W, ALPHA[v])).count("1") for v in range(7)]
        pz = nz(Pz)
        assert [zv + ngz - pz for zv in z] == want
        # the pairs alpha^0|alpha^1, alpha^2|alpha^3, alpha^4|alpha^5 are disjoint
        for a in (0, 2, 4):
            pair = bin(sel(W, ALPHA[a]) | sel(W, ALPHA[a + 1])).count("1")
            assert pair == z[a] + z[a + 1]


@pytest.mark.parametrize("seed", range(60))
def test_flags_never_miss_a_lighter_codeword(seed):
    """With hb a lower bound on the high columns' weight, every sweep holding
    a codeword lighter than wmin is flagged by the single and paired tests."""
    rng = random.Random(1000 + seed)
    g, r1, P = block_state(rng, zero_frac=rng.choice([0.0, 0.2, 0.5]))
    states, truth, _, ngz = sweeps(g, r1, P)
    hi = [[rng.randrange(0, 18) for _ in range(7)] for _ in range(7)]  # high weights
    hb = min(min(r) for r in hi)
    weights = [[LOW - truth[s][v] + hi[s][v] for v in range(7)] for s in range(7)]
    for wmin in range(min(min(r) for r in weights) - 1, 50):
        thz = LOW + hb - wmin - ngz
        for s, (W, Pz) in enumerate(states):
            z = [bin(sel(W, ALPHA[v])).count("1") for v in range(7)]
            pz = nz(Pz)
            single = max(z) - pz > thz
            pairs = [z[0] + z[1], z[2] + z[3], z[4] + z[5], z[6]]
            paired = max(pairs) - pz > thz
            if min(weights[s]) < wmin:
                assert single and paired
            assert paired or not single  # the paired test flags a superset


@pytest.mark.parametrize("seed", range(20))
def test_step_back_recovers_every_sweep(seed):
    """is_block_fix starts from sweep 6's state and undoes digit 1's moves."""
    rng = random.Random(2000 + seed)
    states, _, mv, _ = sweeps(*block_state(rng))
    W, Pz = states[6]
    for s in range(6, -1, -1):
        assert (W, Pz) == states[s]
        if s > 0:
            W, Pz = pl3_xor(W, mv[s - 1][0]), pl3_xor(Pz, mv[s - 1][1])


@pytest.mark.parametrize("seed", range(30))
def test_on_the_spot_and_flagged_counts_find_the_block_minimum(seed):
    """The on-the-spot form (thz tightened after each exact count) and the
    flagged form (one thz for the block, flagged sweeps counted after it,
    from sweep 6 down) return the same minimum, which is the block's true
    minimum whenever that is below the starting wmin."""
    rng = random.Random(3000 + seed)
    g, r1, P = block_state(rng, zero_frac=rng.choice([0.0, 0.2, 0.4]))
    states, truth, mv, ngz = sweeps(g, r1, P)
    hb = rng.randrange(0, 6)
    hi = [[hb + rng.randrange(0, 4) for _ in range(7)] for _ in range(7)]
    weights = [[LOW - truth[s][v] + hi[s][v] for v in range(7)] for s in range(7)]
    true_min = min(min(r) for r in weights)
    thz_base = LOW + hb - ngz

    def exact(s, wmin):
        return min([wmin] + weights[s])

    for start in (true_min, true_min + 1, true_min + 3, 50):
        # on the spot
        wmin = start
        for s, (W, Pz) in enumerate(states):
            z = [bin(sel(W, ALPHA[v])).count("1") for v in range(7)]
            if max(z) - nz(Pz) > thz_base - wmin:
                wmin = exact(s, wmin)
        spot = wmin
        # flagged, counted after the block from sweep 6 down
        thz = thz_base - start
        fl = 0
        for s, (W, Pz) in enumerate(states):
            z = [bin(sel(W, ALPHA[v])).count("1") for v in range(7)]
            if max(z) - nz(Pz) > thz:
                fl |= 1 << s
        wmin = start
        W, Pz = states[6]
        for s in range(6, -1, -1):
            if (fl >> s) & 1:
                assert (W, Pz) == states[s]
                wmin = exact(s, wmin)
            if s > 0:
                W, Pz = pl3_xor(W, mv[s - 1][0]), pl3_xor(Pz, mv[s - 1][1])
        assert spot == wmin == min(start, true_min)
