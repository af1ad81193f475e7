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
(:386-604) and yields, per level, the canonical sets, their max_zeros and the
survivors; `records` renders the reference's JSONL record shapes.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from .canonical import CanonicalDedup
from .distance import DistanceRunner, LaunchConfig, ToricContext
from .tables import N_POINTS, bounding_cube_points, build_eval_matrix, indices_of, pack_canonical


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

    def run(self, max_k: int, targets: dict[int, int], prune_margin: int | None = None):
        """Yields Level objects for k = 2..max_k, keeping every class
        (prune_margin None) or those with d >= targets[k] - prune_margin, as
        the reference's canonical_champion_search does (champion mode)."""
        parents = self.first_level()
        for k in range(2, max_k + 1):
            td = targets.get(k, 1)
            lv = self.level(parents, k, td)
            yield lv
            if prune_margin is None:
                parents = lv.masks
            else:
                keep = max(1, td - prune_margin)
                parents = lv.masks[lv.max_zeros <= N_POINTS - keep]
            if parents.numel() == 0:
                return


def records(level: Level, best_known_d: int) -> list[dict]:
    """The reference's JSONL records for a level (champion_search_canonical.py:536-583):
    champions (d >= best_known_d), one survivor record per class, the sentinel."""
    masks, sets, mz = level.host()
    lattice = bounding_cube_points()
    out = []
    n_champ = 0
    for m, row, z in zip(masks.tolist(), sets.tolist(), mz.tolist()):
        d = N_POINTS - int(z)
        if d >= best_known_d:
            n_champ += 1
            out.append({"name": f"canon_k{level.k}_d{d}", "indices": list(row),
                        "lattice_points": [list(lattice[i]) for i in row], "k": level.k,
                        "max_zeros": int(z), "min_distance": d, "best_known_d": best_known_d,
                        "new_record": d > best_known_d})
    for m in masks.tolist():
        out.append({"type": "survivor", "k": level.k,
                    "packed": pack_canonical(indices_of(int(m)))})
    out.append({"type": "level_complete", "k": level.k, "n_canonical": len(masks),
                "n_champions": n_champ, "n_survivors": len(masks),
                "eval_distance": level.eval_distance, "verified": True})
    return out
