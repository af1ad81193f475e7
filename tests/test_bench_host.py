"""Host logic of bench.py: workload, sharding, CPU baseline and the
max-over-ranks timing of the multi-GPU path (world size 2 over gloo)."""

from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp

import bench


def test_workload_is_seeded_and_shaped():
    a = bench.make_workload(0, 500)
    b = bench.make_workload(0, 500)
    c = bench.make_workload(1, 500)
    assert a == b and a != c
    assert all(6 <= len(s) <= 14 and len(set(s)) == len(s) and s == sorted(s) for s in a)
    assert all(0 <= i < 49 for s in a for i in s)
    hist = bench.k_histogram(a)
    assert set(hist) == set(range(6, 15))


def test_shard_bounds_cover_exactly():
    for n in (0, 1, 7, 10_000):
        for world in (1, 2, 3, 8):
            spans = [bench.shard_bounds(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(spans[i][1] == spans[i + 1][0] for i in range(world - 1))
            sizes = [hi - lo for lo, hi in spans]
            assert max(sizes) - min(sizes) <= 1


def test_cpu_reference_rate_small():
    sets = bench.make_workload(0, 60, 6, 8)
    r = bench.cpu_reference_rate(sets, 1 << 14, per_k=1, threads=2)
    assert r["value"] > 0 and r["kind"] == "port" and r["cores"] == 2


def _worker(rank, world, port, q):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port),
                       "RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    d = bench.Dist()
    d.init("gloo")
    try:
        mx = d.max(float(rank + 1))
        sm = d.sum(float(rank + 1))
        d.barrier()
        q.put((rank, mx, sm))
    finally:
        d.close()


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


@pytest.mark.timeout(120) if hasattr(pytest.mark, "timeout") else (lambda f: f)
def test_max_over_ranks_gloo_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(90)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=5) for _ in range(2))
    assert got == [(0, 2.0, 3.0), (1, 2.0, 3.0)]


def test_launches_per_step_follow_the_level_structure():
    """gpu_launches counts: prep_exact, scan_tasks and the enumeration walk;
    with information sets also prep_infoset, order_codes, levels123 (levels
    1-3), two plan / scan / walk triples (the two parts) per level 4..the last
    level the Griesmer cap leaves (9 for k_max = 14, 11 for 21), and
    finalize_infoset."""
    assert bench.launches_per_step(14, "auto") == 3 + 4 + 6 * 6
    assert bench.launches_per_step(3, "auto") == 3 + 4
    assert bench.launches_per_step(14, "orbit") == 3
    assert bench.launches_per_step(1, "auto") == 3
    assert bench.launches_per_step(21, "infoset") == 3 + 4 + 6 * 8
