"""Canonical BFS over AGL2(F7) classes with the whole level pipeline on the GPU.

The reference builds each level on the host: it expands every survivor by
every absent point (a Python loop, champion_search_canonical.py:496-506),
canonicalises the raw sets in chunks (:312-319), deduplicates them in a Python
set (:337-345), re-batches (:346-350) and evaluates (:353-362).  Here one
level is five device steps with no host round trip but one count:

  tg_expand_canonical   canonical mask of every one-point extension
  tg_hashset_insert     first-occurrence dedup across the whole search
  tg_compact_sets       order-preserving compaction into index rows
  tg_max_zeros          one persistent launch over the level
  (torch compare)       survivors by the keep threshold

`CanonicalBFS.run` drives levels like `canonical_champion_search`
(:386-604) -- targets, prune margin and evaluation mode, sampled screening,
resume -- and yields, per level, the canonical sets and their max_zeros;
`level_records` / `append_records` / `load_canonical_state` write and read
the reference's JSONL results file, so either side resumes the other's run.
"""

from __future__ import annotations

import ctypes
import json
from dataclasses import dataclass
from pathlib import Path

import numpy as np
import torch

from . import _lib
from .canonical import CanonicalDedup
from .distance import DistanceRunner, LaunchConfig, ToricContext
from .tables import (N_POINTS, bounding_cube_points, build_eval_matrix, indices_of, mask_of,
                     pack_canonical, unpack_canonical)


@dataclass
class Level:
    """One BFS level: canonical sets of size k and their evaluation."""

    k: int
    masks: torch.Tensor       # (m,) int64 canonical masks, first-occurrence order
    sets: torch.Tensor        # (m, k) int32 sorted exponent indices
    max_zeros: torch.Tensor   # (m,) int32
    eval_distance: int

    def host(self):
        return (self.masks.cpu().numpy().view(np.uint64), self.sets.cpu().numpy(),
                self.max_zeros.cpu().numpy())


class CanonicalBFS:
    """Level-by-level canonical search on one GPU."""

    def __init__(self, device_id: int = 0, dedup_capacity: int = 1 << 24,
                 config: LaunchConfig | None = None):
        self.device = torch.device("cuda", device_id)
        self.ctx = ToricContext(device_id, build_eval_matrix())
        self.runner = DistanceRunner(self.ctx, config)
        self.dedup = CanonicalDedup(device_id, dedup_capacity)
        self.stream = torch.cuda.Stream(device=self.device)
        self._lib = _lib.load()

    def first_level(self) -> torch.Tensor:
        """The single class of 1-point sets: {0}."""
        return torch.ones(1, dtype=torch.int64, device=self.device)

    def expand(self, parents: torch.Tensor, k_child: int):
        """New canonical classes of size k_child reachable from `parents`
        (int64 canonical masks of size k_child - 1): masks, rows, offsets."""
        lib, s = self._lib, self.stream
        n = parents.numel()
        with torch.cuda.stream(s):
            kids = torch.empty(n * N_POINTS, dtype=torch.int64, device=self.device)
            _lib.check(lib.tg_expand_canonical(self.ctx.handle, parents.data_ptr(), n,
                                               kids.data_ptr(), s.cuda_stream),
                       "tg_expand_canonical")
            is_new, _, status = self.dedup.insert_device(kids, stream=s)
            m_cap = kids.numel()
            scratch_b = ctypes.c_size_t(0)
            _lib.check(lib.tg_compact_scratch_bytes(m_cap, ctypes.byref(scratch_b)),
                       "tg_compact_scratch_bytes")
            scratch = torch.empty(max(int(scratch_b.value), 4), dtype=torch.uint8,
                                  device=self.device)
            out_masks = torch.empty(max(m_cap, 1), dtype=torch.int64, device=self.device)
            out_sets = torch.empty((max(m_cap, 1), k_child), dtype=torch.int32,
                                   device=self.device)
            out_off = torch.empty(max(m_cap, 1) + 1, dtype=torch.int64, device=self.device)
            count = torch.zeros(1, dtype=torch.int32, device=self.device)
            _lib.check(lib.tg_compact_sets(kids.data_ptr(), is_new.data_ptr(), m_cap, k_child,
                                           scratch.data_ptr(), out_masks.data_ptr(),
                                           out_sets.data_ptr(), out_off.data_ptr(),
                                           count.data_ptr(), s.cuda_stream),
                       "tg_compact_sets")
            h = torch.empty(2, dtype=torch.int32, pin_memory=True)
            h[0:1].copy_(count, non_blocking=True)
            h[1:2].copy_(status, non_blocking=True)
        s.synchronize()
        if int(h[1]) == _lib.TG_ERR_CAPACITY:
            raise _lib.ToricLibError(_lib.TG_ERR_CAPACITY, "dedup table more than half full")
        m = int(h[0])
        return out_masks[:m], out_sets[:m], out_off[:m + 1]

    def evaluate(self, sets: torch.Tensor, offsets: torch.Tensor, k: int,
                 target_distance: int) -> torch.Tensor:
        m = sets.shape[0]
        out = torch.empty(max(m, 1), dtype=torch.int32, device=self.device)
        if m:
            p = self.runner.params(m, k, target_distance)
            with torch.cuda.stream(self.stream):
                self.runner.run(p, sets, offsets, out, stream=self.stream)
        return out[:m]

    def level(self, parents: torch.Tensor, k: int, eval_distance: int) -> Level:
        masks, sets, offsets = self.expand(parents, k)
        mz = self.evaluate(sets, offsets, k, eval_distance)
        self.stream.synchronize()
        return Level(k, masks, sets, mz, eval_distance)

    def evaluate_sampled(self, sets: torch.Tensor, offsets: torch.Tensor, k: int,
                         target_distance: int, sample_count: int, sample_seed: int,
                         batch_size: int) -> torch.Tensor:
        """Sampled screening of a level, as the reference's driver batches it:
        set j of the level is position j % batch_size of its batch, the
        sampling id of the reference kernel (blockIdx.x), with the level's
        seed."""
        m = sets.shape[0]
        out = torch.empty(max(m, 1), dtype=torch.int32, device=self.device)
        if m:
            ids = (torch.arange(m, dtype=torch.int32, device=self.device) % batch_size)
            p = self.runner.params(m, k, target_distance, sample_count, sample_seed)
            with torch.cuda.stream(self.stream):
                self.runner.run(p, sets, offsets, out, d_set_ids=ids, stream=self.stream)
        return out[:m]

    def run(self, max_k: int, targets: dict[int, int], prune_margin: int | None = None, *,
            prune_eval_mode: str = "champion", screen_from_k: int | None = None,
            screen_sample_count: int = 0, screen_seed: int = 1, batch_size: int = 50_000,
            results_file: Path | str | None = None, resume: bool = True,
            screen_candidate_log_limit: int = 200, lattice=None,
            keys_file: Path | str | None = None):
        """Yields Level objects for the levels up to max_k, following
        canonical_champion_search (champion_search_canonical.py:386-604):
        per level k the target td = targets[k], keep distance and evaluation
        distance from prune_margin / prune_eval_mode, sampled screening for
        k >= screen_from_k, survivors (every class when prune_margin is None,
        else those with d >= keep distance) as the next level's parents.
        With results_file, the level's records are appended in the
        reference's JSONL format, and a run resumes after the last completed
        level of that file (load_canonical_state).  With keys_file, each
        level is also appended to a binary key stream (append_key_level);
        without a results file, a run resumes from the key stream."""
        if prune_eval_mode not in ("champion", "survivor"):
            raise ValueError("prune_eval_mode must be 'champion' or 'survivor'")
        path = Path(results_file) if results_file is not None else None
        keys_path = Path(keys_file) if keys_file is not None else None
        lattice = lattice if lattice is not None else bounding_cube_points()
        start_k, packed0 = 1, {0}
        if path is not None and resume and path.exists():
            start_k, packed0 = load_canonical_state(path)
        elif keys_path is not None and resume and keys_path.exists():
            start_k, packed0 = load_key_stream_state(keys_path)
        masks0 = sorted(mask_of(unpack_canonical(p, start_k)) for p in packed0)
        parents = torch.tensor(masks0, dtype=torch.int64, device=self.device)
        for k in range(start_k + 1, max_k + 1):
            if parents.numel() == 0:
                return
            td, keep_distance, eval_distance, sample_count = level_settings(
                k, targets, prune_margin, prune_eval_mode, screen_from_k, screen_sample_count)
            masks, sets, offsets = self.expand(parents, k)
            if sample_count > 0:
                mz = self.evaluate_sampled(sets, offsets, k, eval_distance, sample_count,
                                           screen_seed + k * 1_000_003, batch_size)
            else:
                mz = self.evaluate(sets, offsets, k, eval_distance)
            self.stream.synchronize()
            lv = Level(k, masks, sets, mz, eval_distance)
            if path is not None:
                h_masks, _, h_mz = lv.host()
                packed = [pack_canonical(indices_of(int(m))) for m in h_masks.tolist()]
                indices = [indices_of(int(m)) for m in h_masks.tolist()]
                recs, _ = level_records(k, packed, indices, h_mz.tolist(), lattice, td,
                                        prune_margin=prune_margin,
                                        prune_eval_mode=prune_eval_mode,
                                        sample_count=sample_count,
                                        screen_candidate_log_limit=screen_candidate_log_limit)
                append_records(recs, path)
            if keys_path is not None:
                h_masks, _, h_mz = lv.host()
                kept = (np.ones(h_mz.shape, dtype=bool) if prune_margin is None
                        else h_mz <= N_POINTS - keep_distance)
                append_key_level(keys_path, k, h_masks, h_mz, kept, eval_distance=eval_distance,
                                 keep_distance=keep_distance, screened=sample_count > 0)
            yield lv
            if prune_margin is None:
                parents = lv.masks
            else:
                parents = lv.masks[lv.max_zeros <= N_POINTS - keep_distance]


# ---------------------------------------------------------------------------
# The reference's JSONL records (host side)
# ---------------------------------------------------------------------------

def level_settings(k: int, targets: dict[int, int], prune_margin: int | None,
                   prune_eval_mode: str, screen_from_k: int | None,
                   screen_sample_count: int) -> tuple[int, int, int, int]:
    """(td, keep_distance, eval_distance, sample_count) of level k
    (champion_search_canonical.py:479-491)."""
    td = targets.get(k, 1)
    keep_distance = 1 if prune_margin is None else max(1, td - prune_margin)
    eval_distance = td if prune_margin is None or prune_eval_mode == "champion" else keep_distance
    sample_count = screen_sample_count if screen_from_k is not None and k >= screen_from_k else 0
    return td, keep_distance, eval_distance, sample_count


def level_records(k: int, packed, indices, max_zeros, lattice, td: int, *,
                  prune_margin: int | None = None, prune_eval_mode: str = "champion",
                  sample_count: int = 0, screen_candidate_log_limit: int = 200,
                  eval_distance: int | None = None) -> tuple[list[dict], list[int]]:
    """The records canonical_champion_search appends for one level, in its
    order and key order (champion_search_canonical.py:531-583), and the
    packed keys the level keeps as survivors:
      * a champion record per set with d >= td on an exact level;
      * on a screened level instead up to screen_candidate_log_limit
        unverified candidate records;
      * a survivor record per kept set (all sets when prune_margin is None,
        else those with d >= max(1, td - prune_margin));
      * the level_complete sentinel.
    packed, indices and max_zeros are the level's sets in evaluation order;
    eval_distance, when given, is the distance the level was evaluated at
    (else the driver's rule derives it from td and the prune settings)."""
    _, keep_distance, derived_eval, _ = level_settings(k, {k: td}, prune_margin,
                                                       prune_eval_mode, None, 0)
    if eval_distance is None:
        eval_distance = derived_eval
    screened = sample_count > 0
    out: list[dict] = []
    kept: list[int] = []
    seen_kept: set[int] = set()
    n_champ = 0
    n_logged = 0
    for p, S, mz in zip(packed, indices, max_zeros):
        mz = int(mz)
        d = N_POINTS - mz
        S = [int(i) for i in S]
        if d >= td and not screened:
            n_champ += 1
            out.append({"name": f"canon_k{k}_d{d}", "indices": S,
                        "lattice_points": [list(lattice[i]) for i in S], "k": k,
                        "max_zeros": mz, "min_distance": d, "best_known_d": td,
                        "new_record": d > td})
        elif d >= td and screened and n_logged < screen_candidate_log_limit:
            n_logged += 1
            out.append({"type": "candidate", "verified": False,
                        "name": f"screen_k{k}_sample_d{d}", "indices": S,
                        "lattice_points": [list(lattice[i]) for i in S], "k": k,
                        "sampled_max_zeros": mz, "sampled_min_distance": d, "best_known_d": td,
                        "sample_count": sample_count})
        if prune_margin is None or d >= keep_distance:
            if p not in seen_kept:
                seen_kept.add(p)
                kept.append(p)
            out.append({"type": "survivor", "k": k, "packed": int(p)})
    out.append({"type": "level_complete", "k": k, "n_canonical": len(packed),
                "n_champions": n_champ, "n_survivors": len(kept),
                "prune_eval_mode": prune_eval_mode, "eval_distance": eval_distance,
                "keep_distance": keep_distance, "screen_sample_count": sample_count,
                "verified": not screened})
    return out, kept


def append_records(records, path: Path | str) -> None:
    """Appends records as JSON lines (champion_search_canonical.py:168-170)."""
    with Path(path).open("a") as f:
        for r in records:
            f.write(json.dumps(r) + "\n")


def load_canonical_state(path: Path | str) -> tuple[int, set[int]]:
    """(last completed k, packed survivors of that level) of a results file,
    or (1, {0}) when it holds no completed level -- the resume rule of
    champion_search_canonical.py:190-210, so a device-BFS run and the
    reference driver resume each other's files."""
    path = Path(path)
    survivors: dict[int, set[int]] = {}
    completed: set[int] = set()
    if path.exists():
        for line in path.read_text().splitlines():
            line = line.strip()
            if not line:
                continue
            rec = json.loads(line)
            if rec.get("type") == "level_complete":
                completed.add(rec["k"])
            elif rec.get("type") == "survivor":
                survivors.setdefault(rec["k"], set()).add(rec["packed"])
    if not completed:
        return 1, {0}
    last = max(completed)
    return last, survivors.get(last, set())


def records(level: Level, best_known_d: int, prune_margin: int | None = None,
            prune_eval_mode: str = "champion", sample_count: int = 0) -> list[dict]:
    """The reference's JSONL records of a device-BFS level (level_records on
    its canonical sets, in the level's order)."""
    masks, _, mz = level.host()
    packed = [pack_canonical(indices_of(int(m))) for m in masks.tolist()]
    indices = [indices_of(int(m)) for m in masks.tolist()]
    out, _ = level_records(level.k, packed, indices, mz.tolist(), bounding_cube_points(),
                           best_known_d, prune_margin=prune_margin,
                           prune_eval_mode=prune_eval_mode, sample_count=sample_count,
                           eval_distance=level.eval_distance)
    return out


# ---------------------------------------------------------------------------
# Binary key stream (host side)
# ---------------------------------------------------------------------------
#
# At high k the JSONL results file holds one survivor line per kept class
# (about 40 bytes each, parsed line by line on resume).  The key stream keeps
# the same facts in fixed-width little-endian arrays, one block per level:
#
#   file header   b"TGKS", uint32 version (1)
#   level block   b"LEVL", int32 k, int32 flags (bit 0: values from sampled
#                 screening), int64 n, int32 eval_distance,
#                 int32 keep_distance, n x uint64 canonical masks,
#                 n x int8 max_zeros, n x uint8 kept (survivor) flags,
#                 b"DONE"
#
# A block without its closing b"DONE" (a run stopped while writing it) is
# not a completed level: readers ignore it, as the JSONL reader ignores a
# level without its level_complete record.  The JSONL file stays the
# reference's format; the key stream is an addition next to it.

KEYS_MAGIC = b"TGKS"
KEYS_VERSION = 1
_LEVEL_HEAD = np.dtype([("magic", "S4"), ("k", "<i4"), ("flags", "<i4"), ("n", "<i8"),
                        ("eval_distance", "<i4"), ("keep_distance", "<i4")])


@dataclass
class KeyLevel:
    """One completed level of a key stream."""

    k: int
    masks: np.ndarray        # (n,) uint64 canonical masks, evaluation order
    max_zeros: np.ndarray    # (n,) int8
    kept: np.ndarray         # (n,) bool, survivors for the next level
    eval_distance: int
    keep_distance: int
    screened: bool


def append_key_level(path: Path | str, k: int, masks, max_zeros, kept, *, eval_distance: int,
                     keep_distance: int, screened: bool = False) -> None:
    """Appends one level block (writing the file header first when the file
    is new or empty)."""
    masks = np.ascontiguousarray(np.asarray(masks).astype("<u8", copy=False))
    mz = np.asarray(max_zeros)
    if mz.size and (int(mz.min()) < 0 or int(mz.max()) > N_POINTS):
        raise ValueError("max_zeros must lie in 0..49")
    mz = np.ascontiguousarray(mz.astype("<i1"))
    kept = np.ascontiguousarray(np.asarray(kept, dtype=bool).astype("<u1"))
    if not (masks.shape == mz.shape == kept.shape) or masks.ndim != 1:
        raise ValueError("masks, max_zeros and kept must be 1-D of one length")
    head = np.zeros(1, dtype=_LEVEL_HEAD)
    head[0] = (b"LEVL", k, 1 if screened else 0, masks.size, eval_distance, keep_distance)
    path = Path(path)
    new = not path.exists() or path.stat().st_size == 0
    with path.open("ab") as f:
        if new:
            f.write(KEYS_MAGIC + np.uint32(KEYS_VERSION).astype("<u4").tobytes())
        f.write(head.tobytes())
        f.write(masks.tobytes())
        f.write(mz.tobytes())
        f.write(kept.tobytes())
        f.write(b"DONE")


def read_key_stream(path: Path | str) -> list[KeyLevel]:
    """The completed levels of a key stream, in file order; a trailing
    incomplete block is ignored.  Raises ValueError on a foreign file."""
    data = Path(path).read_bytes()
    if not data:
        return []
    if len(data) < 8 or data[:4] != KEYS_MAGIC:
        raise ValueError(f"{path}: not a key stream")
    version = int(np.frombuffer(data[4:8], dtype="<u4")[0])
    if version != KEYS_VERSION:
        raise ValueError(f"{path}: key stream version {version}, expected {KEYS_VERSION}")
    out: list[KeyLevel] = []
    pos, hs = 8, _LEVEL_HEAD.itemsize
    while pos + hs <= len(data):
        head = np.frombuffer(data[pos:pos + hs], dtype=_LEVEL_HEAD)[0]
        if head["magic"] != b"LEVL":
            raise ValueError(f"{path}: bad level block at byte {pos}")
        n = int(head["n"])
        end = pos + hs + 10 * n + 4
        if n < 0 or end > len(data):
            break  # incomplete block
        body = pos + hs
        masks = np.frombuffer(data[body:body + 8 * n], dtype="<u8").astype(np.uint64)
        mz = np.frombuffer(data[body + 8 * n:body + 9 * n], dtype="<i1").copy()
        kept = np.frombuffer(data[body + 9 * n:body + 10 * n], dtype="<u1").astype(bool)
        if data[end - 4:end] != b"DONE":
            break  # incomplete block
        out.append(KeyLevel(int(head["k"]), masks, mz, kept, int(head["eval_distance"]),
                            int(head["keep_distance"]), bool(int(head["flags"]) & 1)))
        pos = end
    return out


def load_key_stream_state(path: Path | str) -> tuple[int, set[int]]:
    """(last completed k, packed survivors of that level) of a key stream, or
    (1, {0}) when it holds no completed level: the same answer
    load_canonical_state gives for the JSONL file of the same run."""
    path = Path(path)
    levels = read_key_stream(path) if path.exists() else []
    if not levels:
        return 1, {0}
    last = max(lv.k for lv in levels)
    packed: set[int] = set()
    for lv in levels:
        if lv.k == last:
            packed.update(pack_canonical(indices_of(int(m))) for m in lv.masks[lv.kept])
    return last, packed
