"""The device-side canonical BFS (expansion, canonicalisation, dedup,
compaction, evaluation) against exhaustive class counts and the oracle."""

from __future__ import annotations

from itertools import combinations

import numpy as np
import pytest

from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def test_bfs_levels_cover_every_class(canon_oracle, M):
    import torch

    from generalized_toric_gpu_search_b200.search import CanonicalBFS, records
    from generalized_toric_gpu_search_b200.tables import indices_of

    bfs = CanonicalBFS(0, dedup_capacity=1 << 22)
    levels = list(bfs.run(max_k=5, targets={}))
    assert [lv.k for lv in levels] == [2, 3, 4, 5]
    for lv in levels:
        masks, sets, mz = lv.host()
        # every k-subset's class appears exactly once
        all_sets = np.array(list(combinations(range(49), lv.k)), dtype=np.int32)
        classes = set(canon_oracle.compute_masks(all_sets).tolist())
        assert len(masks) == len(set(masks.tolist())) == len(classes)
        assert set(masks.tolist()) == classes
        for m, row in zip(masks.tolist()[:50], sets.tolist()[:50]):
            assert list(indices_of(int(m))) == row
        want = orc.max_zeros_batch(M, sets.tolist(), 1)
        assert mz.tolist() == want
    assert [len(lv.masks) for lv in levels[:2]] == [1, 3]
    recs = records(levels[1], best_known_d=40)
    assert recs[-1] == {"type": "level_complete", "k": 3, "n_canonical": 3, "n_champions":
                        sum(1 for r in recs if "name" in r), "n_survivors": 3,
                        "prune_eval_mode": "champion", "eval_distance": 1,
                        "keep_distance": 1, "screen_sample_count": 0, "verified": True}
    torch.cuda.synchronize()


def test_bfs_pruned_with_targets(M):
    from generalized_toric_gpu_search_b200.search import CanonicalBFS

    bfs = CanonicalBFS(0, dedup_capacity=1 << 22)
    targets = {k: 49 - k + 1 - 3 for k in range(2, 8)}
    seen = []
    for lv in bfs.run(max_k=7, targets=targets, prune_margin=1):
        masks, sets, mz = lv.host()
        td = targets[lv.k]
        exact = orc.max_zeros_batch(M, sets.tolist()[:40], 1)
        for got, e in zip(mz.tolist()[:40], exact):
            if e <= 49 - td:
                assert got == e
            else:
                assert got > 49 - td
        seen.append(len(masks))
    assert seen[0] == 1


def test_bfs_key_stream_matches_levels_and_resumes(tmp_path):
    """CanonicalBFS.run with keys_file writes each level's canonical masks,
    values and survivor flags to the binary key stream; a second run with
    only the key stream resumes after its last level and yields what an
    uninterrupted run yields (every class kept, levels 2..7)."""
    from generalized_toric_gpu_search_b200.search import CanonicalBFS, read_key_stream

    targets = {k: 30 for k in range(2, 8)}
    keys = tmp_path / "keys.bin"
    full = [lv.host() for lv in CanonicalBFS(0, dedup_capacity=1 << 22).run(
        max_k=7, targets=targets)]
    assert len(full) == 6
    first = [lv.host() for lv in CanonicalBFS(0, dedup_capacity=1 << 22).run(
        max_k=5, targets=targets, keys_file=keys)]
    stream = read_key_stream(keys)
    assert [lv.k for lv in stream] == [2, 3, 4, 5]
    for (masks, _, mz), lv in zip(first, stream):
        assert np.array_equal(lv.masks, masks)
        assert np.array_equal(lv.max_zeros.astype(np.int32), mz)
        assert lv.kept.all() and lv.keep_distance == 1
    rest = [lv.host() for lv in CanonicalBFS(0, dedup_capacity=1 << 22).run(
        max_k=7, targets=targets, keys_file=keys)]
    assert [len(r[0]) for r in rest] == [len(f[0]) for f in full[4:]]
    for (m_a, _, z_a), (m_b, _, z_b) in zip(rest, full[4:]):
        assert sorted(zip(m_a.tolist(), z_a.tolist())) == sorted(zip(m_b.tolist(), z_b.tolist()))
    assert [lv.k for lv in read_key_stream(keys)] == [2, 3, 4, 5, 6, 7]


def test_autotune_small_table(tmp_path, gpu_oracle):
    from generalized_toric_gpu_search_b200 import _lib, autotune
    from generalized_toric_gpu_search_b200.distance import DistanceOracleCUDABP
    from generalized_toric_gpu_search_b200.tables import build_eval_matrix

    path = tmp_path / "autotune.json"
    cands = [dict(tail_rows=3, blocks_per_sm=8, threads_per_block=128),
             dict(tail_rows=4, blocks_per_sm=8, threads_per_block=128)]
    table = autotune.tune(0, ks=[9], candidates=cands, path=path)
    assert set(table) == {9} and table[9]["tail_rows"] in (3, 4)
    cfg = autotune.choose(autotune.load_table(_lib.device_info(0)[3], path), 9)
    o = DistanceOracleCUDABP(0, build_eval_matrix(), config=cfg)
    sets = autotune.calibration_sets(9)[:50]
    assert o.max_zeros_batch(sets, 1) == gpu_oracle.max_zeros_batch(sets, 1)
