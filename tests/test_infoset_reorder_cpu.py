"""The column reorder of the information-set preparation
(is_compress_masks / is_compress / is_reorder_columns in
csrc/infoset_kernel.cuh), as a host model against a direct gather.

A set's 49 columns are reordered so that the columns outside its pivot set
come first, in increasing order, and the pivot columns last.  The kernel does
this with two bit compresses per plane (the parallel-suffix compress of
Hacker's Delight, 7-4): six rounds, round i shifting the selected bits right
by 2^i, with move masks that depend on the selection mask only.  This test
restates those rounds on Python integers (64-bit words) and checks them
against a column-by-column gather, on random pivot sets of every size and on
the edge cases (no pivots, every column a pivot, pivots at either end).
"""

from __future__ import annotations

import numpy as np
import pytest

N = 49
MASK49 = (1 << N) - 1
M64 = (1 << 64) - 1


def compress_masks(m: int) -> list[int]:
    """Move masks of the six rounds for selection mask m."""
    mk = (~m << 1) & M64  # the zeros of m to the right of each bit
    out = []
    for i in range(6):
        mp = (mk ^ (mk << 1)) & M64  # parity of those zeros, by a prefix XOR
        for s in (2, 4, 8, 16, 32):
            mp ^= (mp << s) & M64
        mv = mp & m
        out.append(mv)
        m = ((m ^ mv) | (mv >> (1 << i))) & M64
        mk &= ~mp & M64
    return out


def compress(x: int, m: int, mv: list[int]) -> int:
    x &= m
    for i in range(6):
        t = x & mv[i]
        x = (x ^ t) | (t >> (1 << i))
    return x


def reorder(piv: int, plane: int) -> int:
    rest = ~piv & MASK49
    piv &= MASK49
    nr = bin(rest).count("1")
    return compress(plane, rest, compress_masks(rest)) | (
        compress(plane, piv, compress_masks(piv)) << nr)


def reorder_direct(piv: int, plane: int) -> int:
    cols = [c for c in range(N) if not (piv >> c) & 1] + [c for c in range(N) if (piv >> c) & 1]
    return sum(((plane >> c) & 1) << d for d, c in enumerate(cols))


def _mask(cols) -> int:
    m = 0
    for c in cols:
        m |= 1 << int(c)
    return m


@pytest.mark.parametrize("n_piv", [0, 1, 2, 6, 10, 14, 17, 21, 30, 48, 49])
def test_compress_reorder_matches_the_column_gather(n_piv):
    rng = np.random.default_rng(700 + n_piv)
    for _ in range(200):
        piv = _mask(rng.choice(N, n_piv, replace=False))
        for _ in range(3):
            plane = int(rng.integers(0, 1 << 62)) & MASK49
            assert reorder(piv, plane) == reorder_direct(piv, plane)


def test_edge_pivot_sets():
    rng = np.random.default_rng(5)
    planes = [0, MASK49, 1, 1 << 48] + [int(rng.integers(0, 1 << 62)) & MASK49 for _ in range(20)]
    pivs = [0, MASK49, _mask(range(14)), _mask(range(35, 49)), _mask(range(0, 49, 2)),
            _mask([0, 48]), 1, 1 << 48]
    for piv in pivs:
        for plane in planes:
            got = reorder(piv, plane)
            assert got == reorder_direct(piv, plane)
            assert got >> N == 0  # nothing lands above column 48
            assert bin(got).count("1") == bin(plane).count("1")  # weights are kept
