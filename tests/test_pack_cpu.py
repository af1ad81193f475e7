"""Host batch packer (csrc/pack.c) against the numpy packing path.

The max_zeros entry points take a list of index lists
(kernel_cuda_bp.py:290-323); both packers must give the same int32 flat
array, int64 offsets and k_max, including for empty and ragged batches.
"""

from __future__ import annotations

import numpy as np
import pytest

from generalized_toric_gpu_search_b200 import build as lib_build
from generalized_toric_gpu_search_b200 import distance as D


@pytest.fixture(scope="module")
def packer():
    lib_build.build_pack()
    from generalized_toric_gpu_search_b200 import _pack

    return _pack


def _numpy_pack(batch, monkeypatch):
    with monkeypatch.context() as m:
        m.setattr(D, "_PACKER", None)
        return D.pack_sets(batch)


def _same(a, b):
    assert a[0].dtype == b[0].dtype == np.int32
    assert a[1].dtype == b[1].dtype == np.int64
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])
    assert a[2] == b[2]


@pytest.mark.parametrize("batch", [
    [], [[]], [[], []], [[0]], [[48, 0, 17]], [[1, 2], [], [3, 4, 5, 6]],
    [tuple(range(21))], [list(range(49))],
])
def test_edge_batches(packer, monkeypatch, batch):
    monkeypatch.setattr(D, "_PACKER", packer)
    _same(D.pack_sets(batch), _numpy_pack(batch, monkeypatch))


def test_random_ragged(packer, monkeypatch):
    rng = np.random.default_rng(7)
    batch = [rng.choice(49, size=int(rng.integers(0, 22)), replace=False).tolist()
             for _ in range(3000)]
    monkeypatch.setattr(D, "_PACKER", packer)
    got = D.pack_sets(batch)
    _same(got, _numpy_pack(batch, monkeypatch))
    assert got[0].flags.writeable and got[1].flags.writeable


def test_out_of_range_flags(packer):
    flat, off, k_max, bad = packer.pack([[1, 2], [49]])
    assert bad and k_max == 2
    assert np.frombuffer(flat, np.int32).tolist() == [1, 2, 49]
    _, _, _, bad = packer.pack([[0, 48]])
    assert not bad
    # values beyond int32 come back as -1 so a range check rejects them
    flat, _, _, bad = packer.pack([[2**40, 3]])
    assert bad and np.frombuffer(flat, np.int32).tolist() == [-1, 3]


def test_other_element_types_fall_back(packer, monkeypatch):
    monkeypatch.setattr(D, "_PACKER", packer)
    with pytest.raises(TypeError):
        packer.pack([[1.0, 2]])
    flat, off, k = D.pack_sets([[1.0, 2], np.array([3, 4, 5])])
    assert flat.tolist() == [1, 2, 3, 4, 5] and off.tolist() == [0, 2, 5] and k == 3
    with pytest.raises(TypeError):
        packer.pack(5)


def test_pack_into_caller_buffers(packer):
    rng = np.random.default_rng(9)
    batch = [rng.choice(49, size=int(rng.integers(0, 22)), replace=False).tolist()
             for _ in range(500)]
    flat_b, off_b, k_max, bad = packer.pack(batch)
    off_ref = np.frombuffer(off_b, np.int64)
    total = int(off_ref[-1])
    f = np.full(total + 5, -7, np.int32)
    o = np.zeros(len(batch) + 1, np.int64)
    # too small: sizes reported, nothing written past the given capacities
    assert packer.pack_into(batch, f.ctypes.data, total - 1, o.ctypes.data, o.size) == (
        total, k_max, False, False)
    assert (f[total - 1:] == -7).all()
    o[:] = 0
    assert packer.pack_into(batch, f.ctypes.data, f.size, o.ctypes.data, len(batch)) == (
        total, k_max, False, False)
    assert not o.any()
    # enough room: the same arrays as pack()
    assert packer.pack_into(batch, f.ctypes.data, f.size, o.ctypes.data, o.size) == (
        total, k_max, bad, True)
    np.testing.assert_array_equal(f[:total], np.frombuffer(flat_b, np.int32)[:total])
    np.testing.assert_array_equal(o, off_ref)
    assert (f[total:] == -7).all()
    # out-of-range indices are flagged, non-int items raise
    assert packer.pack_into([[1, 50]], f.ctypes.data, f.size, o.ctypes.data, o.size)[2]
    with pytest.raises(TypeError):
        packer.pack_into([[1, "a"]], f.ctypes.data, f.size, o.ctypes.data, o.size)


@pytest.mark.parametrize("batch", [
    [[3, 4], (5, 6, 7)],                        # lists and tuples: the one-pass path
    ((3, 4), [5, 6, 7]),                        # a tuple batch
    [[3, 4], np.array([5, 6, 7])],              # an array set: the general path
    [[3, np.int64(4)], [5, 6, 7]],              # a numpy int in a list
    [[3, True], [5, 6, 7]],                     # a bool (an int subclass)
    [[3, 2**40], [5, -1, 7]],                   # a multi-digit int and a negative one
    [[3, 4], [5, 6, 7]] * 1000,                 # long enough to reach the prefetches
])
def test_pack_into_paths_agree_with_pack(packer, batch):
    """The one-pass path (lists or tuples of exact small ints) and the
    general path write what pack() returns, whichever the batch takes."""
    flat_b, off_b, k_max, bad = packer.pack(batch)
    off_ref = np.frombuffer(off_b, np.int64)
    total = int(off_ref[-1])
    f = np.full(total + 3, -7, np.int32)
    o = np.zeros(len(batch) + 1, np.int64)
    assert packer.pack_into(batch, f.ctypes.data, f.size, o.ctypes.data, o.size) == (
        total, k_max, bad, True)
    np.testing.assert_array_equal(f[:total], np.frombuffer(flat_b, np.int32)[:total])
    np.testing.assert_array_equal(o, off_ref)
    assert (f[total:] == -7).all()


@pytest.fixture
def host_stage(packer, monkeypatch):
    """PinnedBatchStage on a machine without a GPU: pinned allocation becomes
    ordinary allocation (the buffers' contents and sizes are what is tested)."""
    import torch

    real_empty = torch.empty

    def empty(*args, pin_memory=False, **kwargs):
        return real_empty(*args, **kwargs)

    monkeypatch.setattr(torch, "empty", empty)
    monkeypatch.setattr(D, "_PACKER", packer)
    return D.PinnedBatchStage()


def test_stage_pack_grows_and_matches(host_stage):
    rng = np.random.default_rng(10)
    for n in (1, 100, 9000):  # the last one outgrows both initial buffers
        batch = [rng.choice(49, size=int(rng.integers(0, 22)), replace=False).tolist()
                 for _ in range(n)]
        h_idx, h_off, k_max, bad = host_stage.pack(batch)
        flat, offsets, k_ref = D.pack_sets(batch)
        assert not bad and k_max == k_ref
        np.testing.assert_array_equal(h_off.numpy(), offsets)
        np.testing.assert_array_equal(h_idx.numpy()[:flat.size], flat)
        assert h_idx.numel() == max(flat.size, 1)
    assert host_stage.pack([[], []])[0].tolist() == [0]
    assert host_stage.pack([[1.5, 2]]) is None  # non-int items: the caller packs with numpy
    assert host_stage.pack([[7, 49]])[3]  # out of range flagged


def test_stage_pack_arrays(host_stage):
    rng = np.random.default_rng(11)
    arrays = [np.sort(rng.choice(49, size=int(rng.integers(0, 16)), replace=False)).astype(np.int32)
              for _ in range(5000)]
    h_idx, h_off, k_max = host_stage.pack_arrays(arrays)
    flat = np.concatenate(arrays)
    np.testing.assert_array_equal(h_idx.numpy()[:flat.size], flat)
    np.testing.assert_array_equal(h_off.numpy(), np.concatenate([[0], np.cumsum([a.size for a in arrays])]))
    assert k_max == max(a.size for a in arrays)
    h_idx, h_off, k_max = host_stage.pack_arrays([np.zeros(0, np.int32)])
    assert h_idx.tolist() == [0] and h_off.tolist() == [0, 0] and k_max == 0
