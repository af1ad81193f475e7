"""tg_max_zeros_noalloc: max_zeros for callers that cannot allocate device memory.

Some hosts of this library may not call cudaMalloc once they are running --
the device memory belongs to another allocator or was carved out at start-up,
or the caller sits in a latency-bound loop that cannot take an allocation's
implicit synchronisation.  tg_max_zeros_noalloc serves them from a 16 MiB
scratch array built into the library.  These tests call it through the C ABI
and compare every output with the allocating entry point tg_max_zeros on the
same inputs, over consecutive calls (the scratch array keeps the previous
call's contents, so stale state would show up in the second call).

This file is collected last on purpose: if it fails, a run stopped at the first
failure has already run every other test.
"""

from __future__ import annotations

import ctypes
import random

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch

    from generalized_toric_gpu_search_b200 import _lib
    from generalized_toric_gpu_search_b200 import build as lib_build
    from generalized_toric_gpu_search_b200.distance import ToricContext
    from generalized_toric_gpu_search_b200.tables import build_eval_matrix

    if not torch.cuda.is_available():
        pytest.fail("gpu test collected without a CUDA device")
    lib_build.build()
    ctx = ToricContext(0, build_eval_matrix())
    return _lib, _lib.load(), ctx, torch


def _run_both(env, sets, td, sample_count=0, seed=0):
    _lib, lib, ctx, torch = env
    from generalized_toric_gpu_search_b200.distance import pack_sets

    flat, offsets, kmax = pack_sets(sets)
    n = len(sets)
    dev = torch.device("cuda", 0)
    d_idx = torch.from_numpy(flat).to(dev)
    d_off = torch.from_numpy(offsets).to(dev)
    per_set = not np.isscalar(td)
    d_td = torch.tensor(td, dtype=torch.int32, device=dev) if per_set else None
    p = _lib.DistanceParams(n_sets=n, k_max=kmax, target_distance=0 if per_set else td,
                            sample_count=sample_count, sample_seed=seed)
    need = ctypes.c_size_t(0)
    assert lib.tg_distance_workspace_size(ctypes.byref(p), ctypes.byref(need)) == 0
    ws = torch.empty(int(need.value), dtype=torch.uint8, device=dev)
    out_ref = torch.full((n,), -1, dtype=torch.int32, device=dev)
    out_static = torch.full((n,), -2, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    td_ptr = d_td.data_ptr() if per_set else None
    _lib.check(lib.tg_max_zeros(ctx.handle, ctypes.byref(p), d_idx.data_ptr(), d_off.data_ptr(),
                                td_ptr, None, out_ref.data_ptr(), ws.data_ptr(), ws.numel(),
                                stream), "tg_max_zeros")
    _lib.check(lib.tg_max_zeros_noalloc(ctx.handle, ctypes.byref(p), d_idx.data_ptr(),
                                        d_off.data_ptr(), td_ptr, None, out_static.data_ptr(),
                                        stream), "tg_max_zeros_noalloc")
    torch.cuda.synchronize()
    return out_ref.cpu().tolist(), out_static.cpu().tolist()


def test_noalloc_matches_allocating_entry_point(env):
    rng = random.Random(77)
    # first call: a larger exact batch of mixed k
    sets1 = [sorted(rng.sample(range(49), rng.randint(2, 11))) for _ in range(400)]
    a, b = _run_both(env, sets1, 1)
    assert a == b
    # second call in a row: fewer sets, per-set thresholds (early exits); the
    # scratch still holds the first call's tables and abort flags
    sets2 = [sorted(rng.sample(range(49), rng.randint(3, 9))) for _ in range(60)]
    tds = [rng.randint(20, 45) for _ in sets2]
    a, b = _run_both(env, sets2, tds)
    for x, y, td in zip(a, b, tds):
        assert (x > 49 - td) == (y > 49 - td)
        if x <= 49 - td:
            assert x == y
    # third call: sampled screening, bit-exact across the two entry points
    sets3 = [sorted(rng.sample(range(49), rng.randint(5, 30))) for _ in range(50)]
    a, b = _run_both(env, sets3, 1, sample_count=4096, seed=123)
    assert a == b


def test_noalloc_rejects_oversized_batch(env):
    _lib, lib, ctx, torch = env
    p = _lib.DistanceParams(n_sets=1_000_000, k_max=21, target_distance=1)
    dummy = torch.zeros(8, dtype=torch.int64, device="cuda")
    st = lib.tg_max_zeros_noalloc(ctx.handle, ctypes.byref(p), dummy.data_ptr(),
                                  dummy.data_ptr(), None, None, dummy.data_ptr(), None)
    assert st == _lib.TG_ERR_WORKSPACE
    assert "static workspace" in _lib.last_error()


def test_noalloc_out_of_range_set_reads_zero(env):
    """A set with an index outside 0..48 comes back as 0 from the zero-allocation
    entry point (it has no status query); the other sets of the batch keep the
    values a clean batch gives them.  The allocating entry point gives the
    same values (and reports the set through tg_distance_status)."""
    rng = random.Random(91)
    clean = [sorted(rng.sample(range(49), rng.randint(3, 10))) for _ in range(30)]
    bad = [list(s) for s in clean]
    bad[7] = bad[7][:-1] + [49]
    bad[19] = [-1] + bad[19][1:]
    want, want_static = _run_both(env, clean, 1)
    assert want == want_static
    got, got_static = _run_both(env, bad, 1)
    for i in range(len(clean)):
        if i in (7, 19):
            assert got[i] == 0 and got_static[i] == 0
        else:
            assert got[i] == want[i] and got_static[i] == want[i]
