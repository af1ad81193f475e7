"""Failure handling of the device-resident request loop, made on the host.

No GPU is faulted or hung: a malformed request, a full slot pool, a full
host queue, a cancelled request, admission without enough device memory,
and a publication that never arrives (tg_server_debug_skip_publication,
after which the loop's bounded wait for it runs out and reports
TG_ERR_STATE) -- each checked to end in a clear error while the server keeps
answering the other requests correctly.
"""

from __future__ import annotations

import ctypes
import random
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = 49


def _check(answers, sets, exact, td=1):
    tmax = N - td
    for a, s, e in zip(answers, sets, exact):
        if e <= tmax:
            assert a.passed and a.max_zeros == e, s
        else:
            assert not a.passed and a.max_zeros > tmax, s


def test_malformed_requests(gpu_oracle):
    from generalized_toric_gpu_search_b200.serve import ToricServer

    with ToricServer(0, k_max=12, max_slots=16) as srv:
        with pytest.raises(ValueError):
            srv.submit([0, 49], 1)
        with pytest.raises(ValueError):
            srv.submit([-3, 4], 1)
        with pytest.raises(ValueError):
            srv.submit(list(range(13)), 1)
        rng = random.Random(1)
        sets = [sorted(rng.sample(range(N), 10)) for _ in range(20)]
        _check(srv.evaluate([(s, 1) for s in sets], timeout=120), sets,
               gpu_oracle.max_zeros_batch(sets, 1))


def test_full_slot_pool_through_the_abi(gpu_oracle, M):
    """tg_server_submit refuses with TG_ERR_CAPACITY while every slot holds an
    unanswered request, and accepts again once answers free them."""
    import torch

    from generalized_toric_gpu_search_b200 import _lib
    from generalized_toric_gpu_search_b200.distance import ToricContext

    lib = _lib.load()
    ctx = ToricContext(0, M)
    p = _lib.ServerParams(max_slots=2, k_max=12, table_capacity=-1)
    slots, dev_b, host_b = ctypes.c_int32(0), ctypes.c_size_t(0), ctypes.c_size_t(0)
    _lib.check(lib.tg_server_layout(ctx.handle, ctypes.byref(p), ctypes.byref(slots),
                                    ctypes.byref(dev_b), ctypes.byref(host_b)), "layout")
    assert slots.value == 2
    arena = torch.empty(int(dev_b.value), dtype=torch.uint8, device="cuda")
    host = torch.empty(int(host_b.value), dtype=torch.uint8, pin_memory=True)
    h = ctypes.c_void_p()
    _lib.check(lib.tg_server_create(ctx.handle, ctypes.byref(p), arena.data_ptr(), arena.numel(),
                                    host.data_ptr(), host.numel(), ctypes.byref(h)), "create")
    rng = random.Random(2)
    sets = [sorted(rng.sample(range(N), 9)) for _ in range(3)]
    rid = ctypes.c_uint32(0)
    for s in sets[:2]:
        arr = np.array(s, dtype=np.int32)
        assert lib.tg_server_submit(h, arr.ctypes.data, len(s), 1, ctypes.byref(rid)) == 0
    arr = np.array(sets[2], dtype=np.int32)
    assert lib.tg_server_submit(h, arr.ctypes.data, 9, 1, ctypes.byref(rid)) == \
        _lib.TG_ERR_CAPACITY
    assert "busy" in _lib.last_error()
    out = (_lib.ServerResult * 4)()
    got = {}
    running = ctypes.c_int32(0)
    deadline = time.time() + 60
    while len(got) < 2 and time.time() < deadline:
        _lib.check(lib.tg_server_pump(h, ctypes.byref(running)), "pump")
        n = ctypes.c_int32(0)
        _lib.check(lib.tg_server_poll(h, out, 4, ctypes.byref(n)), "poll")
        for i in range(n.value):
            got[int(out[i].id)] = int(out[i].max_zeros)
        time.sleep(0.001)
    assert sorted(got.values()) == sorted(gpu_oracle.max_zeros_batch(sets[:2], 1))
    assert lib.tg_server_submit(h, arr.ctypes.data, 9, 1, ctypes.byref(rid)) == 0
    deadline = time.time() + 60
    while len(got) < 3 and time.time() < deadline:
        _lib.check(lib.tg_server_pump(h, ctypes.byref(running)), "pump")
        n = ctypes.c_int32(0)
        _lib.check(lib.tg_server_poll(h, out, 4, ctypes.byref(n)), "poll")
        for i in range(n.value):
            got[int(out[i].id)] = int(out[i].max_zeros)
        time.sleep(0.001)
    assert got[int(rid.value)] == gpu_oracle.max_zeros_batch(sets[2:], 1)[0]
    _lib.check(lib.tg_server_destroy(h), "destroy")


def test_full_host_queue_and_cancellation(gpu_oracle):
    from generalized_toric_gpu_search_b200 import _lib
    from generalized_toric_gpu_search_b200.serve import ToricServer

    rng = random.Random(3)
    sets = [sorted(rng.sample(range(N), 14)) for _ in range(40)]
    with ToricServer(0, k_max=15, max_slots=1, max_pending=8) as srv:
        futs = []
        with pytest.raises(_lib.ToricLibError) as err:
            for s in sets:
                futs.append(srv.submit(s, 1))
        assert err.value.status == _lib.TG_ERR_CAPACITY
        assert 8 <= len(futs) < len(sets)
        cancelled = [srv.cancel(f) for f in futs[2:]]
        assert any(cancelled)
        for f, c in zip(futs[2:], cancelled):
            assert f.cancelled() == c
        kept = [(s, f) for s, f in zip(sets, futs) if not f.cancelled()]
        answers = [f.result(timeout=120) for _, f in kept]
        _check(answers, [s for s, _ in kept], gpu_oracle.max_zeros_batch([s for s, _ in kept], 1))
        assert not srv.cancel(futs[0])  # answered already


def test_admission_without_device_memory():
    from generalized_toric_gpu_search_b200 import _lib
    from generalized_toric_gpu_search_b200.serve import ToricServer

    with pytest.raises(_lib.ToricLibError) as err:
        ToricServer(0, k_max=15, memory_fraction=1e-12)
    assert err.value.status == _lib.TG_ERR_CAPACITY
    assert "free device memory" in str(err.value)


def test_missing_publication_times_out_and_the_loop_goes_on(gpu_oracle):
    """The loop waits a bounded time for a publication entry; when the entry
    never comes it records TG_ERR_STATE and serves the next requests."""
    from generalized_toric_gpu_search_b200 import _lib
    from generalized_toric_gpu_search_b200.serve import ToricServer

    rng = random.Random(4)
    sets = [sorted(rng.sample(range(N), 11)) for _ in range(30)]
    exact = gpu_oracle.max_zeros_batch(sets, 1)
    with ToricServer(0, k_max=12, max_slots=32) as srv:
        _check(srv.evaluate([(s, 1) for s in sets[:10]], timeout=120), sets[:10], exact[:10])
        assert srv.stats()["device_status"] == 0
        _lib.check(_lib.load().tg_server_debug_skip_publication(srv.handle), "skip")
        _check(srv.evaluate([(s, 1) for s in sets[10:]], timeout=120), sets[10:], exact[10:])
        # The later requests may all be answered before the wait for the
        # missing entry (a few milliseconds) runs out: poll the status.
        deadline = time.time() + 5.0
        st = srv.stats()
        while st["device_status"] == 0 and time.time() < deadline:
            time.sleep(0.002)
            st = srv.stats()
    assert st["device_status"] == _lib.TG_ERR_STATE
    assert st["published"] == 31 and st["finished"] == 30


def test_submit_many_is_all_or_none(gpu_oracle):
    """submit_many queues a list in one step or, when the host queue would
    overflow or a request is malformed, queues none of it."""
    from generalized_toric_gpu_search_b200 import _lib
    from generalized_toric_gpu_search_b200.serve import ToricServer

    rng = random.Random(9)
    sets = [sorted(rng.sample(range(N), 12)) for _ in range(12)]
    with ToricServer(0, k_max=15, max_slots=1, max_pending=6) as srv:
        with pytest.raises(_lib.ToricLibError) as err:
            srv.submit_many([(s, 1) for s in sets])
        assert err.value.status == _lib.TG_ERR_CAPACITY
        with pytest.raises(ValueError):
            srv.submit_many([(sets[0], 1), ([0, 49], 1)])
        assert srv.stats()["published"] == 0
        futs = srv.submit_many([(s, 1) for s in sets[:5]])
        _check([f.result(timeout=120) for f in futs], sets[:5],
               gpu_oracle.max_zeros_batch(sets[:5], 1))


def test_batch_submission_through_the_c_abi(M, gpu_oracle):
    """tg_server_submit_batch takes requests in order under one lock: a
    malformed one gets its own error status and no id, the slots' end stops
    the batch (the rest stay with the caller), and every accepted request
    gets the batch oracle's answer."""
    import torch

    from generalized_toric_gpu_search_b200 import _lib
    from generalized_toric_gpu_search_b200.distance import ToricContext

    lib = _lib.load()
    ctx = ToricContext(0, M)
    p = _lib.ServerParams(max_slots=3, k_max=12, table_capacity=-1)
    slots, dev_b, host_b = ctypes.c_int32(0), ctypes.c_size_t(0), ctypes.c_size_t(0)
    _lib.check(lib.tg_server_layout(ctx.handle, ctypes.byref(p), ctypes.byref(slots),
                                    ctypes.byref(dev_b), ctypes.byref(host_b)), "layout")
    arena = torch.empty(int(dev_b.value), dtype=torch.uint8, device="cuda")
    host = torch.empty(int(host_b.value), dtype=torch.uint8, pin_memory=True)
    h = ctypes.c_void_p()
    _lib.check(lib.tg_server_create(ctx.handle, ctypes.byref(p), arena.data_ptr(), arena.numel(),
                                    host.data_ptr(), host.numel(), ctypes.byref(h)), "create")
    rng = random.Random(21)
    good = [sorted(rng.sample(range(N), 9)) for _ in range(4)]
    reqs = [good[0], [3, 60, 7], good[1], good[2], good[3]]  # the second is malformed
    flat = np.array([i for s in reqs for i in s], dtype=np.int32)
    offs = np.zeros(len(reqs) + 1, dtype=np.int64)
    offs[1:] = np.cumsum([len(s) for s in reqs])
    td = np.ones(len(reqs), dtype=np.int32)
    ids = np.zeros(len(reqs), dtype=np.uint32)
    st = np.full(len(reqs), 99, dtype=np.int32)
    consumed = ctypes.c_int32(-1)
    _lib.check(lib.tg_server_submit_batch(h, flat.ctypes.data, offs.ctypes.data, len(reqs),
                                          td.ctypes.data, ids.ctypes.data, st.ctypes.data,
                                          ctypes.byref(consumed)), "submit_batch")
    # three slots: good[0], the malformed one (no slot), good[1], good[2]; good[3] waits
    assert consumed.value == 4
    assert st[:4].tolist() == [0, _lib.TG_ERR_INVALID_ARGUMENT, 0, 0]
    want = dict(zip([int(ids[0]), int(ids[2]), int(ids[3])],
                    gpu_oracle.max_zeros_batch([good[0], good[1], good[2]], 1)))
    out = (_lib.ServerResult * 4)()
    got = {}
    running = ctypes.c_int32(0)
    deadline = time.time() + 60
    while len(got) < 3 and time.time() < deadline:
        _lib.check(lib.tg_server_pump(h, ctypes.byref(running)), "pump")
        n = ctypes.c_int32(0)
        _lib.check(lib.tg_server_poll(h, out, 4, ctypes.byref(n)), "poll")
        for i in range(n.value):
            got[int(out[i].id)] = int(out[i].max_zeros)
        time.sleep(0.001)
    assert got == want
    _lib.check(lib.tg_server_destroy(h), "destroy")
