"""AGL2(F7) canonical forms and canonical dedup on the B200.

`CanonicalOracle` keeps the interface of kernel_canon.py:133-191
(`CanonicalOracle(device_id, gl2_perms, rel_table).compute(sets)` returning an
object array of Python ints `lo | hi << 64`, k <= 16) and `init_canon_oracle`.
`compute_masks` extends it to any set size with the 49-bit canonical mask,
and `CanonicalDedup` keeps a device hash set of canonical masks (the `seen`
set of champion_search_canonical.py:312-345, on the device).
"""

from __future__ import annotations

import ctypes
import threading

import numpy as np
import torch

from . import _lib
from .distance import ToricContext, _require_cuda
from .tables import N_POINTS, build_eval_matrix, precompute_gl2_perms
from .tables import rel_table as _difference_table

MAX_KEY_K = 16


class CanonicalOracle:
    """GPU canonical-form engine; one instance per CUDA device.

    The signature is the reference's, `CanonicalOracle(device_id, gl2_perms,
    rel_table)` (kernel_canon.py:137-142), positionally or by keyword.
    `gl2_perms` and `rel_table` are accepted for interface compatibility and
    checked against the tables the library builds itself.  `rel_table_arr`
    is an older keyword-only spelling of `rel_table`."""

    def __init__(self, device_id: int, gl2_perms: np.ndarray | None = None,
                 rel_table: np.ndarray | None = None, *,
                 rel_table_arr: np.ndarray | None = None):
        _require_cuda(device_id)
        rel = _pick_rel_table(rel_table, rel_table_arr)
        if gl2_perms is not None and not np.array_equal(np.asarray(gl2_perms),
                                                        precompute_gl2_perms()):
            raise ValueError("gl2_perms differs from GL2(F7) on the 49 exponent points")
        if rel is not None and not np.array_equal(np.asarray(rel), _difference_table()):
            raise ValueError("rel_table differs from the Z_7^2 difference table")
        self.device_id = device_id
        self.ctx = ToricContext(device_id, build_eval_matrix())
        self.device = torch.device("cuda", device_id)
        self._stream = torch.cuda.Stream(device=self.device)
        self._lock = threading.Lock()

    def compute_device(self, d_sets: torch.Tensor, k: int, stream: torch.cuda.Stream | None = None,
                       with_keys: bool = True):
        """Device-level: (n, k) int32 CUDA tensor -> (mask, key_lo, key_hi, status) tensors."""
        n = d_sets.shape[0] if d_sets.dim() == 2 else d_sets.numel() // max(k, 1)
        st = stream if stream is not None else torch.cuda.current_stream(self.device)
        out_mask = torch.empty(n, dtype=torch.int64, device=self.device)
        lo = torch.empty(n, dtype=torch.int64, device=self.device) if with_keys else None
        hi = torch.empty(n, dtype=torch.int64, device=self.device) if with_keys else None
        status = torch.zeros(1, dtype=torch.int32, device=self.device)
        _lib.check(
            _lib.load().tg_canonical_sets(
                self.ctx.handle, d_sets.data_ptr() if k > 0 else None, n, k,
                out_mask.data_ptr(), lo.data_ptr() if lo is not None else None,
                hi.data_ptr() if hi is not None else None, status.data_ptr(), st.cuda_stream,
            ),
            "tg_canonical_sets",
        )
        return out_mask, lo, hi, status

    def _run_sets(self, sets: np.ndarray):
        arr = np.ascontiguousarray(np.asarray(sets, dtype=np.int32))
        if arr.ndim != 2:
            raise ValueError("sets must be an (n, k) array")
        n, k = arr.shape
        if k > N_POINTS:
            raise ValueError("a set has at most 49 points")
        if arr.size and (int(arr.min()) < 0 or int(arr.max()) >= N_POINTS):
            raise ValueError("exponent indices must lie in 0..48")
        with self._lock, torch.cuda.device(self.device):
            s = self._stream
            with torch.cuda.stream(s):
                src = arr if arr.size else np.zeros((max(n, 1), 1), np.int32)
                d_sets = torch.from_numpy(src).pin_memory().to(self.device, non_blocking=True)
                mask, lo, hi, status = self.compute_device(d_sets, k, stream=s)
                h = torch.empty((4, n), dtype=torch.int64, pin_memory=True)
                h[0].copy_(mask, non_blocking=True)
                h[1].copy_(lo, non_blocking=True)
                h[2].copy_(hi, non_blocking=True)
                h_st = torch.empty(1, dtype=torch.int32, pin_memory=True)
                h_st.copy_(status, non_blocking=True)
            s.synchronize()
        if int(h_st[0]) != _lib.TG_OK:
            raise ValueError("canonical form: a row repeats an index or leaves 0..48")
        u = h[:3].numpy().view(np.uint64)
        return u[0].copy(), u[1].copy(), u[2].copy()

    def compute(self, sets: np.ndarray) -> np.ndarray:
        """(n, k) int32 rows -> (n,) object array of packed keys lo + hi * 2**64."""
        arr = np.asarray(sets)
        if arr.ndim != 2:
            raise ValueError("sets must be an (n, k) array")
        n, k = arr.shape
        if k > MAX_KEY_K:
            raise ValueError("GPU canonical kernel supports k <= 16")
        if n == 0:
            return np.zeros(0, dtype=object)
        _, lo, hi = self._run_sets(arr)
        return keys_from_words(lo, hi)

    def compute_masks(self, sets) -> np.ndarray:
        """Rows of any size 1..49 (or an (n,) array of 49-bit masks as uint64)
        -> (n,) uint64 canonical masks."""
        arr = np.asarray(sets)
        if arr.ndim == 1 and arr.dtype in (np.uint64, np.int64):
            return self.canonical_masks_from_masks(arr.astype(np.uint64))
        if arr.ndim != 2 or arr.shape[0] == 0:
            return np.zeros(0 if arr.ndim != 2 else arr.shape[0], dtype=np.uint64)
        mask, _, _ = self._run_sets(arr)
        return mask

    def canonical_masks_from_masks(self, masks: np.ndarray) -> np.ndarray:
        m = np.ascontiguousarray(np.asarray(masks, dtype=np.uint64))
        n = m.shape[0]
        if n == 0:
            return np.zeros(0, dtype=np.uint64)
        with self._lock, torch.cuda.device(self.device):
            s = self._stream
            with torch.cuda.stream(s):
                d_in = torch.from_numpy(m.view(np.int64)).pin_memory().to(self.device,
                                                                           non_blocking=True)
                out = torch.empty(n, dtype=torch.int64, device=self.device)
                _lib.check(_lib.load().tg_canonical_masks(self.ctx.handle, d_in.data_ptr(), n,
                                                          out.data_ptr(), None, None,
                                                          s.cuda_stream),
                           "tg_canonical_masks")
                h = torch.empty(n, dtype=torch.int64, pin_memory=True)
                h.copy_(out, non_blocking=True)
            s.synchronize()
        return h.numpy().view(np.uint64).copy()


def _pick_rel_table(rel_table, rel_table_arr):
    if rel_table is not None and rel_table_arr is not None:
        raise TypeError("pass rel_table or rel_table_arr, not both")
    return rel_table if rel_table is not None else rel_table_arr


def keys_from_words(lo: np.ndarray, hi: np.ndarray) -> np.ndarray:
    """(n,) object array of the Python ints lo + hi * 2**64, the form of the
    reference's keys (kernel_canon.py:174-176).  The high word is zero up to
    k = 11, so only the rows that have one pay for the wide arithmetic (half
    the host time of a million k <= 10 keys)."""
    out = np.asarray(lo, dtype=np.uint64).astype(object)
    hi = np.asarray(hi, dtype=np.uint64)
    nz = np.flatnonzero(hi)
    if nz.size:
        out[nz] = out[nz] + (hi[nz].astype(object) << 64)
    return out


def init_canon_oracle(device_id: int, gl2_perms: np.ndarray | None = None,
                      rel_table: np.ndarray | None = None, *,
                      rel_table_arr: np.ndarray | None = None) -> CanonicalOracle:
    """Builds a CanonicalOracle (kernel_canon.py:179-191).  The reference's
    driver calls it as init_canon_oracle(device_id=..., gl2_perms=...,
    rel_table=...) (champion_search_canonical.py:447-451)."""
    rel = _pick_rel_table(rel_table, rel_table_arr)
    _, _, _, name = _lib.device_info(device_id)
    print(f"[canon] GPU {device_id}: {name} — canonical kernel ready")
    return CanonicalOracle(device_id, gl2_perms, rel)


class CanonicalDedup:
    """Device hash set of 64-bit canonical keys with first-occurrence semantics."""

    def __init__(self, device_id: int, capacity: int = 1 << 20):
        _require_cuda(device_id)
        cap = 64
        while cap < capacity:
            cap <<= 1
        self.capacity = cap
        self.device = torch.device("cuda", device_id)
        nbytes = ctypes.c_size_t(0)
        _lib.check(_lib.load().tg_hashset_bytes(cap, ctypes.byref(nbytes)), "tg_hashset_bytes")
        self.table = torch.empty(int(nbytes.value), dtype=torch.uint8, device=self.device)
        self.call_id = 0
        self.clear()

    def clear(self, stream: torch.cuda.Stream | None = None) -> None:
        st = stream if stream is not None else torch.cuda.current_stream(self.device)
        _lib.check(_lib.load().tg_hashset_clear(self.table.data_ptr(), self.capacity,
                                                st.cuda_stream), "tg_hashset_clear")
        self.call_id = 0

    def insert_device(self, d_keys: torch.Tensor, stream: torch.cuda.Stream | None = None):
        """Inserts int64/uint64 keys; returns (is_new uint8, n_new int32, status int32) tensors."""
        st = stream if stream is not None else torch.cuda.current_stream(self.device)
        n = d_keys.numel()
        self.call_id += 1
        is_new = torch.empty(max(n, 1), dtype=torch.uint8, device=self.device)
        n_new = torch.zeros(1, dtype=torch.int32, device=self.device)
        status = torch.zeros(1, dtype=torch.int32, device=self.device)
        _lib.check(_lib.load().tg_hashset_insert(self.table.data_ptr(), self.capacity,
                                                 d_keys.data_ptr(), n, self.call_id,
                                                 is_new.data_ptr(), n_new.data_ptr(),
                                                 status.data_ptr(), st.cuda_stream),
                   "tg_hashset_insert")
        return is_new[:n], n_new, status

    def insert(self, keys: np.ndarray) -> np.ndarray:
        """Host convenience: bool array, True where a key is new (first occurrence)."""
        k = np.ascontiguousarray(np.asarray(keys, dtype=np.uint64)).view(np.int64)
        with torch.cuda.device(self.device):
            d = torch.from_numpy(k).to(self.device)
            is_new, _, status = self.insert_device(d)
            out = is_new.cpu().numpy().astype(bool)
            st = int(status.item())
        if st == _lib.TG_ERR_CAPACITY:
            raise _lib.ToricLibError(st, "canonical dedup table is more than half full")
        if st != _lib.TG_OK:
            _lib.check(st, "tg_hashset_insert (device)")
        return out
