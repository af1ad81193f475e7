"""Autotuner cache and shape selection (host logic, no GPU)."""

from __future__ import annotations

from generalized_toric_gpu_search_b200 import autotune


def test_table_roundtrip_and_choice(tmp_path):
    path = tmp_path / "autotune.json"
    table = {8: dict(tail_rows=3, blocks_per_sm=8, threads_per_block=128),
             12: dict(tail_rows=4, blocks_per_sm=4, threads_per_block=256),
             14: dict(tail_rows=5, blocks_per_sm=8, threads_per_block=128)}
    autotune.save_table("NVIDIA B200", table, path)
    autotune.save_table("other GPU", {6: dict(tail_rows=2, blocks_per_sm=4,
                                               threads_per_block=64)}, path)
    got = autotune.load_table("NVIDIA B200", path)
    assert got == table
    assert autotune.load_table("missing", path) == {}
    assert autotune.choose(got, 13).tail_rows == 4
    assert autotune.choose(got, 14).tail_rows == 5
    assert autotune.choose(got, 21).threads_per_block == 128
    assert autotune.choose(got, 6).tail_rows == 3       # below the smallest tuned k
    assert autotune.choose({}, 10) is None


def test_calibration_batches_are_seeded():
    a = autotune.calibration_sets(10)
    b = autotune.calibration_sets(10)
    assert a == b and all(len(s) == 10 for s in a)
    assert 148 <= len(a) <= 4096
    assert all(c["tail_rows"] in (3, 4, 5) for c in autotune.CANDIDATES)
