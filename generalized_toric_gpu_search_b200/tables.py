"""Host-side constant tables of the toric setting (built once, tiny).

These mirror the reference helpers that callers of the oracles use to build
their inputs: the evaluation matrix (precompute.py:17-43), the GL2(F7) point
permutations and relative-position table (champion_search_canonical.py:61-108)
and the canonical-key decoder (champion_search_canonical.py:153-161).
"""

from __future__ import annotations

import numpy as np

N_POINTS = 49
POLY = 0b1011  # x^3 + x + 1 (gf8.py:9)


def gf8_mul(a: int, b: int) -> int:
    """Product in GF(8) = GF(2)[x]/(x^3 + x + 1)."""
    acc = 0
    while b:
        if b & 1:
            acc ^= a
        b >>= 1
        a <<= 1
        if a & 0b1000:
            a ^= POLY
    return acc


MUL_TABLE = np.array([[gf8_mul(a, b) for b in range(8)] for a in range(8)], dtype=np.uint8)


def gf8_pow(base: int, exp: int) -> int:
    out = 1
    for _ in range(exp):
        out = gf8_mul(out, base)
    return out


def torus_points() -> list[tuple[int, int]]:
    """The 49 points (x, y) of (GF(8)*)^2, column order of M."""
    return [(1 + j // 7, 1 + j % 7) for j in range(N_POINTS)]


def bounding_cube_points() -> list[tuple[int, int]]:
    """Exponent points (a, b) in [0, 6]^2; index i is (i // 7, i % 7)."""
    return [(i // 7, i % 7) for i in range(N_POINTS)]


def eval_monomial(a: tuple[int, int], p: tuple[int, int]) -> int:
    """x^a0 y^a1 at the torus point p = (x, y) (precompute.py:27-29)."""
    return gf8_mul(gf8_pow(p[0], a[0]), gf8_pow(p[1], a[1]))


def build_eval_matrix() -> np.ndarray:
    """49 x 49 int32 matrix: row a*7+b is x^a y^b at the torus points."""
    m = np.zeros((N_POINTS, N_POINTS), dtype=np.int32)
    for i, a in enumerate(bounding_cube_points()):
        for j, p in enumerate(torus_points()):
            m[i, j] = eval_monomial(a, p)
    return m


def precompute_gl2_perms() -> np.ndarray:
    """(2016, 49) int32: GL2(F7) matrices (a b; c d), lexicographic in
    (a, b, c, d), as permutations of the point indices."""
    x = np.arange(N_POINTS) // 7
    y = np.arange(N_POINTS) % 7
    rows = []
    for a in range(7):
        for b in range(7):
            for c in range(7):
                for d in range(7):
                    if (a * d - b * c) % 7:
                        rows.append(((a * x + b * y) % 7) * 7 + (c * x + d * y) % 7)
    return np.asarray(rows, dtype=np.int32)


def rel_table() -> np.ndarray:
    """(49, 49) uint8: entry [p, q] is the index of point q - point p mod 7."""
    a = np.arange(N_POINTS) // 7
    b = np.arange(N_POINTS) % 7
    return (((a[None, :] - a[:, None]) % 7) * 7 + (b[None, :] - b[:, None]) % 7).astype(np.uint8)


def unpack_canonical(packed: int, k: int) -> tuple[int, ...]:
    """Sorted exponent indices of a packed canonical key (6 bits each; for
    k >= 11 index 0 is implicit and the key starts at the second index)."""
    if k <= 10:
        return tuple((packed >> (6 * i)) & 63 for i in range(k))
    return (0,) + tuple((packed >> (6 * i)) & 63 for i in range(k - 1))


def pack_canonical(indices) -> int:
    """Inverse of unpack_canonical for a sorted index tuple containing 0."""
    idx = sorted(int(i) for i in indices)
    k = len(idx)
    start = 0 if k <= 10 else 1
    out = 0
    for pos in range(start, k):
        out |= idx[pos] << (6 * (pos - start))
    return out


def mask_of(indices) -> int:
    m = 0
    for i in indices:
        m |= 1 << int(i)
    return m


def indices_of(mask: int) -> tuple[int, ...]:
    return tuple(i for i in range(N_POINTS) if mask >> i & 1)
