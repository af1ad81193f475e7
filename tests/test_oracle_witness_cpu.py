"""The oracle's witness check (or_codeword_message): given a set S and a
codeword c, it solves m M[S] = c over GF(8), re-evaluates m M[S] and counts
the zeros of c.  Checked here on random messages (the message comes back
exactly, as the toric rows are independent), on vectors outside the code, on
the zero codeword of an independent and of a dependent set of rows."""

from __future__ import annotations

import random

import numpy as np
import pytest

from oracle import oracle as orc


def test_recovers_random_messages(M):
    mul = orc.mul_table()
    rng = random.Random(1)
    for _ in range(300):
        k = rng.randint(1, 21)
        S = rng.sample(range(49), k)
        m = [rng.randrange(8) for _ in range(k)]
        if not any(m):
            m[0] = 1
        cw = np.zeros(49, dtype=np.int64)
        for c, s in zip(m, S):
            cw ^= mul[c][M[s]]
        zeros, msg = orc.codeword_message(M, S, cw)
        assert zeros == int((cw == 0).sum())
        assert msg == m


def test_rejects_vectors_outside_the_code(M):
    rng = random.Random(2)
    for _ in range(50):
        S = rng.sample(range(49), rng.randint(1, 12))
        cw = np.zeros(49, dtype=np.uint8)
        cw[rng.randrange(49)] = rng.randint(1, 7)
        with pytest.raises(ValueError):
            orc.codeword_message(M, S, cw)


def test_zero_codeword(M):
    with pytest.raises(ValueError):
        orc.codeword_message(M, [0, 1, 2], np.zeros(49))
    M2 = M.copy()
    M2[5] = M2[3]
    zeros, msg = orc.codeword_message(M2, [3, 5, 7], np.zeros(49))
    assert zeros == 49 and any(msg)
