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


def test_concurrent_saves_leave_a_complete_table(tmp_path):
    """Ranks of a multi-GPU run save their tables at the same time: every
    save renames its own temporary file, so the table file is always whole."""
    import multiprocessing as mp

    from generalized_toric_gpu_search_b200 import autotune

    path = tmp_path / "autotune.json"
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_save_many, args=(str(path), r)) for r in range(4)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    table = autotune.load_table("GPU", path)
    assert table and all(v["is_tasks_per_thread"] == 4 for v in table.values())
    assert not list(tmp_path.glob("*.tmp"))


def _save_many(path, rank):
    from pathlib import Path

    from generalized_toric_gpu_search_b200 import autotune

    for i in range(50):
        autotune.save_table("GPU", {6 + (i + rank) % 9: {"is_tasks_per_thread": 4}}, Path(path))
