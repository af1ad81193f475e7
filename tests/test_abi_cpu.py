"""The C-ABI library loads, exports exactly what include/toric_b200.h declares,
and validates arguments without touching a GPU."""

from __future__ import annotations

import ctypes
import re
from pathlib import Path

import pytest

from generalized_toric_gpu_search_b200 import _lib
from generalized_toric_gpu_search_b200 import build as lib_build

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def lib():
    lib_build.build()
    return _lib.load()


def header_symbols() -> set[str]:
    text = (ROOT / "include" / "toric_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b(tg_[a-z0-9_]+)\s*\(", text))


def test_header_matches_bindings(lib):
    declared = header_symbols()
    assert declared == set(_lib.SIGNATURES), declared ^ set(_lib.SIGNATURES)
    for name in declared:
        assert hasattr(lib, name), name


def test_status_strings(lib):
    assert lib.tg_status_string(0) == b"TG_OK"
    assert lib.tg_status_string(7) == b"TG_ERR_BAD_INPUT"
    assert lib.tg_abi_version() == 2
    # tg_distance_params grew by the information-set walk's launch knobs
    assert ctypes.sizeof(_lib.DistanceParams) == 64


def test_device_count_without_gpu(lib):
    n = ctypes.c_int32(-1)
    assert lib.tg_device_count(ctypes.byref(n)) == 0
    assert n.value >= 0


def _ws(lib, **kw):
    p = _lib.DistanceParams(**kw)
    out = ctypes.c_size_t(0)
    return lib.tg_distance_workspace_size(ctypes.byref(p), ctypes.byref(out)), out.value


def test_workspace_size_and_validation(lib):
    st, nbytes = _ws(lib, n_sets=10_000, k_max=14)
    assert st == 0 and nbytes > 10_000 * 40
    st2, nbytes2 = _ws(lib, n_sets=20_000, k_max=14)
    assert st2 == 0 and nbytes2 > nbytes
    assert _ws(lib, n_sets=1, k_max=22)[0] == _lib.TG_ERR_INVALID_ARGUMENT
    assert _ws(lib, n_sets=1, k_max=49, sample_count=10)[0] == 0
    assert _ws(lib, n_sets=1, k_max=50, sample_count=10)[0] == _lib.TG_ERR_INVALID_ARGUMENT
    assert _ws(lib, n_sets=-1, k_max=3)[0] == _lib.TG_ERR_INVALID_ARGUMENT
    assert _ws(lib, n_sets=1, k_max=3, tail_rows=1)[0] == _lib.TG_ERR_INVALID_ARGUMENT
    assert _ws(lib, n_sets=1, k_max=3, threads_per_block=96)[0] == _lib.TG_ERR_INVALID_ARGUMENT
    assert "k <= 21" in _lib.last_error() or "threads_per_block" in _lib.last_error()
    assert _ws(lib, n_sets=1, k_max=3, enumeration=4)[0] == _lib.TG_ERR_INVALID_ARGUMENT
    assert "enumeration" in _lib.last_error()
    # information-set sections: none for orbit-only runs, none for AUTO below
    # its threshold
    st_o, orbit_b = _ws(lib, n_sets=1000, k_max=14, enumeration=_lib.TG_ENUM_ORBIT)
    st_i, infoset_b = _ws(lib, n_sets=1000, k_max=14, enumeration=_lib.TG_ENUM_INFOSET)
    st_a, auto_b = _ws(lib, n_sets=1000, k_max=14)
    assert st_o == st_i == st_a == 0
    assert infoset_b > orbit_b + 1000 * 14 * 8 * 3 and auto_b > orbit_b
    below = _lib.TG_INFOSET_AUTO_MIN_K - 1
    assert _ws(lib, n_sets=1000, k_max=below)[1] == \
        _ws(lib, n_sets=1000, k_max=below, enumeration=_lib.TG_ENUM_ORBIT)[1]


def test_hashset_validation(lib):
    out = ctypes.c_size_t(0)
    assert lib.tg_hashset_bytes(1 << 20, ctypes.byref(out)) == 0
    assert out.value == 256 + 16 * (1 << 20)
    assert lib.tg_hashset_bytes(1000, ctypes.byref(out)) == _lib.TG_ERR_INVALID_ARGUMENT


def test_null_context_rejected(lib):
    p = _lib.DistanceParams(n_sets=1, k_max=3)
    st = lib.tg_max_zeros(None, ctypes.byref(p), None, None, None, None, None, None, 0, None)
    assert st == _lib.TG_ERR_INVALID_ARGUMENT
    st = lib.tg_canonical_sets(None, None, 1, 3, None, None, None, None, None)
    assert st == _lib.TG_ERR_INVALID_ARGUMENT


def test_context_without_device(lib):
    import numpy as np

    from generalized_toric_gpu_search_b200.tables import build_eval_matrix

    n = ctypes.c_int32(0)
    lib.tg_device_count(ctypes.byref(n))
    if n.value:
        pytest.skip("a GPU is visible")
    m = np.ascontiguousarray(build_eval_matrix())
    h = ctypes.c_void_p()
    st = lib.tg_context_create(0, m.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                               ctypes.byref(h))
    assert st == _lib.TG_ERR_NO_DEVICE
    with pytest.raises(RuntimeError, match="No CUDA GPU found"):
        _lib.check(st, "tg_context_create")


def test_infoset_last_level_matches_the_griesmer_cap():
    """The information-set walk's level cap (tg_infoset_last_level) against a
    Python restatement: after level L a k-row toric code's unseen codewords
    weigh >= ceil(49 (L + 1) / k); the Griesmer bound caps d of a [49, k]
    code over GF(8)."""
    import bench

    lib_build.build()
    lib = _lib.load()
    out = ctypes.c_int32(0)
    for k_max in range(0, 22):
        assert lib.tg_infoset_last_level(k_max, 1, ctypes.byref(out)) == 0
        assert out.value == bench.last_infoset_level(k_max)
        assert lib.tg_infoset_last_level(k_max, 0, ctypes.byref(out)) == 0
        assert out.value == k_max
    lib.tg_infoset_last_level(14, 1, ctypes.byref(out))
    assert out.value == 9
    assert lib.tg_infoset_last_level(22, 1, ctypes.byref(out)) == _lib.TG_ERR_INVALID_ARGUMENT
