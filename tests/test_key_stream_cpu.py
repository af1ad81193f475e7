"""The binary key stream of the device BFS (search.append_key_level /
read_key_stream / load_key_stream_state), on the CPU: round trips, an
interrupted last block, foreign files, and agreement with the JSONL records
and resume state of the same level."""

from __future__ import annotations

import numpy as np
import pytest

from generalized_toric_gpu_search_b200 import search
from generalized_toric_gpu_search_b200.tables import (bounding_cube_points, indices_of, mask_of,
                                                      pack_canonical)


def _level(rng, k, n):
    """n distinct k-point masks that contain point 0 (as canonical forms do)."""
    out = set()
    while len(out) < n:
        rest = rng.choice(np.arange(1, 49), k - 1, replace=False)
        out.add(mask_of([0, *rest.tolist()]))
    masks = np.array(sorted(out), dtype=np.uint64)
    mz = rng.integers(20, 40, size=n).astype(np.int32)
    return masks, mz


def test_round_trip_of_several_levels(tmp_path):
    rng = np.random.default_rng(3)
    p = tmp_path / "keys.bin"
    want = []
    for k, n in ((4, 7), (5, 30), (6, 0), (7, 12)):
        masks, mz = _level(rng, k, n) if n else (np.zeros(0, np.uint64), np.zeros(0, np.int32))
        kept = mz <= 30
        search.append_key_level(p, k, masks, mz, kept, eval_distance=19, keep_distance=19,
                                screened=k == 7)
        want.append((k, masks, mz, kept))
    got = search.read_key_stream(p)
    assert [g.k for g in got] == [w[0] for w in want]
    for g, (k, masks, mz, kept) in zip(got, want):
        assert g.masks.dtype == np.uint64 and np.array_equal(g.masks, masks)
        assert np.array_equal(g.max_zeros.astype(np.int32), mz)
        assert np.array_equal(g.kept, kept)
        assert (g.eval_distance, g.keep_distance, g.screened) == (19, 19, k == 7)
    # 8-byte header, 28-byte level head, 10 bytes per set, 4-byte close
    assert p.stat().st_size == 8 + sum(28 + 10 * len(w[1]) + 4 for w in want)


def test_interrupted_last_block_is_not_a_completed_level(tmp_path):
    rng = np.random.default_rng(5)
    p = tmp_path / "keys.bin"
    m4, z4 = _level(rng, 4, 9)
    m5, z5 = _level(rng, 5, 11)
    search.append_key_level(p, 4, m4, z4, np.ones(9, bool), eval_distance=1, keep_distance=1)
    search.append_key_level(p, 5, m5, z5, np.ones(11, bool), eval_distance=1, keep_distance=1)
    data = p.read_bytes()
    for cut in (1, 4, 20, 60):
        q = tmp_path / f"cut{cut}.bin"
        q.write_bytes(data[:-cut])
        got = search.read_key_stream(q)
        assert [g.k for g in got] == [4]
        last, packed = search.load_key_stream_state(q)
        assert last == 4 and packed == {pack_canonical(indices_of(int(m))) for m in m4}


def test_foreign_and_empty_files(tmp_path):
    assert search.load_key_stream_state(tmp_path / "absent.bin") == (1, {0})
    (tmp_path / "empty.bin").write_bytes(b"")
    assert search.read_key_stream(tmp_path / "empty.bin") == []
    (tmp_path / "x.jsonl").write_text('{"type": "level_complete", "k": 3}\n')
    with pytest.raises(ValueError):
        search.read_key_stream(tmp_path / "x.jsonl")
    with pytest.raises(ValueError):
        search.append_key_level(tmp_path / "bad.bin", 3, np.zeros(2, np.uint64),
                                np.array([1, 60]), np.ones(2, bool), eval_distance=1,
                                keep_distance=1)


def test_key_stream_state_equals_the_jsonl_state_of_the_same_levels(tmp_path):
    """The two files written for the same levels resume to the same state:
    load_key_stream_state on the key stream and load_canonical_state on the
    reference's JSONL records (level_records keeps d >= td - margin)."""
    rng = np.random.default_rng(11)
    keys, jsonl = tmp_path / "keys.bin", tmp_path / "results.jsonl"
    td, margin = 22, 2
    for k in (5, 6):
        masks, mz = _level(rng, k, 40)
        _, keep_distance, eval_distance, _ = search.level_settings(k, {k: td}, margin,
                                                                   "champion", None, 0)
        kept = mz <= 49 - keep_distance
        search.append_key_level(keys, k, masks, mz, kept, eval_distance=eval_distance,
                                keep_distance=keep_distance)
        packed = [pack_canonical(indices_of(int(m))) for m in masks.tolist()]
        indices = [indices_of(int(m)) for m in masks.tolist()]
        recs, kept_packed = search.level_records(k, packed, indices, mz.tolist(),
                                                 bounding_cube_points(), td, prune_margin=margin)
        search.append_records(recs, jsonl)
        assert set(kept_packed) == {p for p, f in zip(packed, kept) if f}
    assert search.load_key_stream_state(keys) == search.load_canonical_state(jsonl)
    assert keys.stat().st_size < jsonl.stat().st_size
