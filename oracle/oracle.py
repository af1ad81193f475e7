"""ORACLE — test infrastructure only (tests/, __graft_entry__.smoke() checker,
bench.py CPU-baseline leg).  Never imported by the product package.

Python side of the CPU restatement in toric_oracle.c (see its header for the
reference file:line each function follows), plus pure-Python brute force for
tiny cases, restating the reference's smoke-test brute force
`bf_max_zeros` (kernel backup.py:203-222) and `canonical_forms_batch`
(champion_search_canonical.py:115-140).
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import c_int, c_int64, c_uint64, c_void_p
from pathlib import Path

import numpy as np

ORACLE_DIR = Path(__file__).resolve().parent
SRC = ORACLE_DIR / "toric_oracle.c"
LIB = ORACLE_DIR / "liboracle_toric.so"
NP = 49

_lib = None


def build(force: bool = False) -> Path:
    """gcc -O3 -fopenmp build of the C restatement (portable x86-64-v3)."""
    if not force and LIB.exists() and LIB.stat().st_mtime >= SRC.stat().st_mtime:
        return LIB
    tmp = str(LIB) + f".{os.getpid()}.tmp"  # processes started together may build at once
    cmd = ["gcc", "-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared", "-o", tmp,
           str(SRC)]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + proc.stderr)
    os.replace(tmp, LIB)
    return LIB


def load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        lib = ctypes.CDLL(str(LIB))
        lib.or_max_zeros_batch.restype = c_int
        lib.or_max_zeros_batch.argtypes = [c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_int,
                                           c_int64, c_uint64, c_void_p, c_void_p, c_int]
        lib.or_eval_messages.restype = c_int
        lib.or_eval_messages.argtypes = [c_void_p, c_void_p, c_int, c_uint64, c_uint64]
        lib.or_eval_prefix_batch.restype = c_int64
        lib.or_eval_prefix_batch.argtypes = [c_void_p, c_void_p, c_void_p, c_int, c_uint64, c_int,
                                             c_void_p]
        lib.or_codeword_message.restype = c_int
        lib.or_codeword_message.argtypes = [c_void_p, c_void_p, c_int, c_void_p, c_void_p]
        lib.or_canonical_keys.restype = None
        lib.or_canonical_keys.argtypes = [c_void_p, c_int, c_int, c_void_p, c_void_p, c_int]
        lib.or_canonical_masks.restype = None
        lib.or_canonical_masks.argtypes = [c_void_p, c_int, c_void_p, c_int]
        lib.or_gl2_perms.restype = None
        lib.or_gl2_perms.argtypes = [c_void_p]
        lib.or_rel_table.restype = None
        lib.or_rel_table.argtypes = [c_void_p]
        lib.or_mul_table.restype = None
        lib.or_mul_table.argtypes = [c_void_p]
        _lib = lib
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(c_void_p) if a is not None else None


# ---- tables ----------------------------------------------------------------

def mul_table() -> np.ndarray:
    out = np.zeros(64, dtype=np.int32)
    load().or_mul_table(_ptr(out))
    return out.reshape(8, 8)


def gl2_perms() -> np.ndarray:
    out = np.zeros((2016, NP), dtype=np.int32)
    load().or_gl2_perms(_ptr(out))
    return out


def rel_table() -> np.ndarray:
    out = np.zeros((NP, NP), dtype=np.uint8)
    load().or_rel_table(_ptr(out))
    return out


def eval_matrix() -> np.ndarray:
    """precompute.py:32-43 restated: M[a*7+b, j] = x^a y^b at (1+j//7, 1+j%7)."""
    mul = mul_table()

    def pw(base, e):
        r = 1
        for _ in range(e):
            r = int(mul[r, base])
        return r

    M = np.zeros((NP, NP), dtype=np.int32)
    for i in range(NP):
        for j in range(NP):
            M[i, j] = mul[pw(1 + j // 7, i // 7), pw(1 + j % 7, i % 7)]
    return M


# ---- max_zeros ---------------------------------------------------------------

def max_zeros_batch(M, batched, target_distance=1, sample_count=0, sample_seed=0, set_ids=None,
                    threads=0) -> list[int]:
    """kernel.py:97-203 semantics (see toric_oracle.c)."""
    M = np.ascontiguousarray(np.asarray(M, dtype=np.int32))
    n = len(batched)
    if n == 0:
        return []
    lengths = np.array([len(s) for s in batched], dtype=np.int64)
    offsets = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(lengths, out=offsets[1:])
    flat = np.array([i for s in batched for i in s] or [0], dtype=np.int32)
    td = None
    td_default = 0
    if np.isscalar(target_distance):
        td_default = int(target_distance)
    else:
        td = np.ascontiguousarray(np.asarray(target_distance, dtype=np.int32))
    ids = None if set_ids is None else np.ascontiguousarray(np.asarray(set_ids, dtype=np.int32))
    out = np.zeros(n, dtype=np.int32)
    rc = load().or_max_zeros_batch(_ptr(M), _ptr(flat), _ptr(offsets), n, _ptr(td), td_default,
                                   int(sample_count), int(sample_seed) & (2**64 - 1), _ptr(ids),
                                   _ptr(out), int(threads))
    if rc != 0:
        raise RuntimeError("oracle allocation failed")
    return out.tolist()


def eval_messages(M, S, first: int, count: int) -> int:
    M = np.ascontiguousarray(np.asarray(M, dtype=np.int32))
    s = np.ascontiguousarray(np.asarray(S, dtype=np.int32))
    return load().or_eval_messages(_ptr(M), _ptr(s), len(S), first, count)


def eval_prefix_batch(M, batched, count: int, threads: int = 0) -> tuple[int, list[int]]:
    """Messages 1..min(count, 8^k-1) of every set, no early exit, on `threads`
    OpenMP threads; returns (messages evaluated, max zeros seen per set)."""
    M = np.ascontiguousarray(np.asarray(M, dtype=np.int32))
    n = len(batched)
    lengths = np.array([len(s) for s in batched], dtype=np.int64)
    offsets = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(lengths, out=offsets[1:])
    flat = np.array([i for s in batched for i in s] or [0], dtype=np.int32)
    out = np.zeros(max(n, 1), dtype=np.int32)
    msgs = load().or_eval_prefix_batch(_ptr(M), _ptr(flat), _ptr(offsets), n, int(count),
                                       int(threads), _ptr(out))
    if msgs < 0:
        raise RuntimeError("oracle allocation failed")
    return int(msgs), out[:n].tolist()


def codeword_message(M, S, codeword) -> tuple[int, list[int]]:
    """Checks a witness codeword of the code M[S]: returns (zeros, message)
    with message . M[S] == codeword recomputed by the oracle, or raises
    ValueError when the codeword is not in the code (or is the zero codeword
    of a code whose rows are independent)."""
    M = np.ascontiguousarray(np.asarray(M, dtype=np.int32))
    s = np.ascontiguousarray(np.asarray(S, dtype=np.int32))
    cw = np.ascontiguousarray(np.asarray(codeword, dtype=np.uint8).reshape(NP))
    msg = np.zeros(max(len(S), 1), dtype=np.int32)
    z = load().or_codeword_message(_ptr(M), _ptr(s), len(S), _ptr(cw), _ptr(msg))
    if z < 0:
        raise ValueError(f"not a codeword of the set's code (status {z})")
    return int(z), msg[:len(S)].tolist()


def bf_max_zeros(S, M) -> int:
    """Pure-Python exhaustive max_zeros (kernel backup.py:203-222 semantics)."""
    mul = mul_table()
    k = len(S)
    best = 0
    for pid in range(1, 8 ** k):
        coeffs = [(pid >> (3 * i)) & 7 for i in range(k)]
        z = 0
        for j in range(NP):
            v = 0
            for c, s in zip(coeffs, S):
                v ^= int(mul[c, M[s, j]])
            if v == 0:
                z += 1
        best = max(best, z)
    return best


# ---- canonical forms -----------------------------------------------------------

def canonical_keys(sets: np.ndarray, threads: int = 0) -> list[int]:
    """kernel_canon.py packed keys (lo + hi << 64) for rows of k <= 16."""
    arr = np.ascontiguousarray(np.asarray(sets, dtype=np.int32))
    n, k = arr.shape
    lo = np.zeros(n, dtype=np.uint64)
    hi = np.zeros(n, dtype=np.uint64)
    load().or_canonical_keys(_ptr(arr), n, k, _ptr(lo), _ptr(hi), int(threads))
    return [int(a) | (int(b) << 64) for a, b in zip(lo, hi)]


def canonical_masks(masks, threads: int = 0) -> np.ndarray:
    arr = np.ascontiguousarray(np.asarray(masks, dtype=np.uint64))
    out = np.zeros(arr.shape[0], dtype=np.uint64)
    load().or_canonical_masks(_ptr(arr), arr.shape[0], _ptr(out), int(threads))
    return out


def canonical_forms_numpy(sets_arr: np.ndarray) -> np.ndarray:
    """Vectorised numpy canonical keys for k <= 10 (the reference's CPU path,
    champion_search_canonical.py:115-140, restated)."""
    sets_arr = np.asarray(sets_arr, dtype=np.int32)
    n, k = sets_arr.shape
    if k > 10:
        raise ValueError("CPU canonical fallback supports k <= 10")
    perms = gl2_perms()
    rt = rel_table()
    best = np.full(n, np.iinfo(np.uint64).max, dtype=np.uint64)
    for start in range(0, len(perms), 64):
        img = perms[start:start + 64][:, sets_arr]          # (c, n, k)
        for t in range(k):
            rel = rt[img[:, :, t:t + 1], img]               # (c, n, k)
            rel.sort(axis=2)
            packed = np.zeros(rel.shape[:2], dtype=np.uint64)
            for j in range(k):
                packed |= rel[:, :, j].astype(np.uint64) << np.uint64(6 * j)
            np.minimum(best, packed.min(axis=0), out=best)
    return best
