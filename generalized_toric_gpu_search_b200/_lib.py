"""ctypes binding of libtoric_b200.so (include/toric_b200.h).

The shared library is loaded from the package directory.  There is no CPU
fallback: when the library or a CUDA device is missing, the oracle classes
raise instead of computing anything on the host.
"""

from __future__ import annotations

import ctypes
import threading
from ctypes import POINTER, c_char_p, c_double, c_int, c_int32, c_int64, c_size_t, c_uint32
from ctypes import c_uint64, c_void_p
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libtoric_b200.so"

TG_OK = 0
TG_ERR_INVALID_ARGUMENT = 1
TG_ERR_CUDA = 2
TG_ERR_WORKSPACE = 3
TG_ERR_NO_DEVICE = 4
TG_ERR_CAPACITY = 5
TG_ERR_TIMEOUT = 6
TG_ERR_BAD_INPUT = 7
TG_ERR_STATE = 8

TG_ENUM_AUTO = 0
TG_ENUM_PROJECTIVE = 1
TG_ENUM_ORBIT = 2
TG_ENUM_INFOSET = 3
TG_INFOSET_AUTO_MIN_K = 2
TG_WALK_ENUMERATION = 1
TG_WALK_INFOSET = 2
TG_VARIANT_AUTO = 0
TG_VARIANT_HISTOGRAM = 1
TG_VARIANT_DIRECT = 2

# Every symbol include/toric_b200.h declares, with (restype, argtypes).
SIGNATURES: dict[str, tuple] = {
    "tg_status_string": (c_char_p, [c_int]),
    "tg_last_error": (c_char_p, []),
    "tg_abi_version": (c_int, []),
    "tg_device_count": (c_int, [POINTER(c_int32)]),
    "tg_device_info": (
        c_int,
        [c_int, POINTER(c_int32), POINTER(c_int32), POINTER(c_int32), c_char_p, c_int32],
    ),
    "tg_context_create": (c_int, [c_int, POINTER(c_int32), POINTER(c_void_p)]),
    "tg_context_destroy": (c_int, [c_void_p]),
    "tg_context_is_toric": (c_int, [c_void_p, POINTER(c_int32)]),
    "tg_distance_workspace_size": (c_int, [c_void_p, POINTER(c_size_t)]),
    "tg_max_zeros": (
        c_int,
        [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
         c_size_t, c_void_p],
    ),
    "tg_max_zeros_prepare": (
        c_int,
        [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
         c_size_t, c_void_p],
    ),
    "tg_max_zeros_walk": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_size_t, c_void_p]),
    "tg_max_zeros_walk_part": (
        c_int, [c_void_p, c_void_p, c_int32, c_void_p, c_void_p, c_size_t, c_void_p]
    ),
    "tg_infoset_last_level": (c_int, [c_int32, c_int32, POINTER(c_int32)]),
    "tg_witness_workspace_size": (c_int, [c_void_p, POINTER(c_size_t)]),
    "tg_max_zeros_witness": (
        c_int,
        [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
         c_void_p, c_size_t, c_void_p],
    ),
    "tg_max_zeros_noalloc": (
        c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]
    ),
    "tg_distance_status": (c_int, [c_void_p, c_void_p, c_void_p, POINTER(c_int32)]),
    "tg_distance_counters": (
        c_int,
        [c_void_p, c_void_p, c_void_p, POINTER(c_uint64), POINTER(c_uint64), POINTER(c_double)],
    ),
    "tg_distance_path_counters": (c_int, [c_void_p, c_void_p, c_void_p, POINTER(c_uint64)]),
    "tg_distance_stage_counters": (
        c_int,
        [c_void_p, c_void_p, c_void_p, POINTER(c_uint64), c_int32],
    ),
    "tg_canonical_sets": (
        c_int,
        [c_void_p, c_void_p, c_int32, c_int32, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p],
    ),
    "tg_canonical_masks": (
        c_int, [c_void_p, c_void_p, c_int32, c_void_p, c_void_p, c_void_p, c_void_p]
    ),
    "tg_expand_canonical": (c_int, [c_void_p, c_void_p, c_int32, c_void_p, c_void_p]),
    "tg_compact_scratch_bytes": (c_int, [c_int32, POINTER(c_size_t)]),
    "tg_compact_sets": (
        c_int,
        [c_void_p, c_void_p, c_int32, c_int32, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
         c_void_p],
    ),
    "tg_hashset_bytes": (c_int, [c_int64, POINTER(c_size_t)]),
    "tg_hashset_clear": (c_int, [c_void_p, c_int64, c_void_p]),
    "tg_hashset_insert": (
        c_int,
        [c_void_p, c_int64, c_void_p, c_int32, c_uint32, c_void_p, c_void_p, c_void_p, c_void_p],
    ),
    "tg_measure_int_pipes": (c_int, [c_int, c_void_p, POINTER(c_double)]),
    "tg_server_layout": (
        c_int, [c_void_p, c_void_p, POINTER(c_int32), POINTER(c_size_t), POINTER(c_size_t)]
    ),
    "tg_server_create": (
        c_int, [c_void_p, c_void_p, c_void_p, c_size_t, c_void_p, c_size_t, POINTER(c_void_p)]
    ),
    "tg_server_submit": (c_int, [c_void_p, c_void_p, c_int32, c_int32, POINTER(c_uint32)]),
    "tg_server_submit_batch": (
        c_int,
        [c_void_p, c_void_p, c_void_p, c_int32, c_void_p, c_void_p, c_void_p, POINTER(c_int32)],
    ),
    "tg_server_pump": (c_int, [c_void_p, POINTER(c_int32)]),
    "tg_server_poll": (c_int, [c_void_p, c_void_p, c_int32, POINTER(c_int32)]),
    "tg_server_stats": (c_int, [c_void_p, POINTER(c_uint64)]),
    "tg_server_destroy": (c_int, [c_void_p]),
    "tg_server_debug_skip_publication": (c_int, [c_void_p]),
}

TG_RESULT_PASS = 1
TG_RESULT_FAIL = 2
TG_RESULT_DEDUP = 4
TG_RESULT_BAD_INPUT = 8


class ServerParams(ctypes.Structure):
    """Mirror of tg_server_params."""

    _fields_ = [
        ("max_slots", c_int32),
        ("k_max", c_int32),
        ("tail_rows", c_int32),
        ("blocks_per_sm", c_int32),
        ("idle_us", c_int32),
        ("life_ms", c_int32),
        ("table_capacity", c_int64),
        ("memory_fraction", c_double),
    ]


class ServerResult(ctypes.Structure):
    """Mirror of tg_server_result."""

    _fields_ = [
        ("id", c_uint32),
        ("max_zeros", c_int32),
        ("flags", c_int32),
        ("pad", c_int32),
        ("t_admit_ns", c_uint64),
        ("t_done_ns", c_uint64),
    ]


class DistanceParams(ctypes.Structure):
    """Mirror of tg_distance_params."""

    _fields_ = [
        ("n_sets", c_int32),
        ("k_max", c_int32),
        ("tail_rows", c_int32),
        ("enumeration", c_int32),
        ("variant", c_int32),
        ("blocks_per_sm", c_int32),
        ("threads_per_block", c_int32),
        ("target_distance", c_int32),
        ("sample_count", c_int64),
        ("sample_seed", c_uint64),
        ("is_blocks_per_sm", c_int32),
        ("is_tasks_per_thread", c_int32),
        ("is_max_task_units", c_int32),
        ("is_pad", c_int32),
    ]


class ToricLibError(RuntimeError):
    """A libtoric_b200 call returned a status other than TG_OK."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


_lock = threading.Lock()
_lib: ctypes.CDLL | None = None


def load() -> ctypes.CDLL:
    """Loads the in-tree shared library (raises when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not LIB_PATH.exists():
                raise ImportError(
                    f"{LIB_PATH.name} is missing; build it with "
                    "`python -m generalized_toric_gpu_search_b200.build`"
                )
            lib = ctypes.CDLL(str(LIB_PATH))
            for name, (restype, argtypes) in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = restype
                fn.argtypes = argtypes
            _lib = lib
    return _lib


def last_error() -> str:
    msg = load().tg_last_error()
    return msg.decode() if msg else ""


def check(status: int, what: str) -> None:
    """Raises the Python exception matching a tg_* status."""
    if status == TG_OK:
        return
    lib = load()
    name = lib.tg_status_string(status).decode()
    msg = f"{what}: {name}: {last_error()}"
    if status in (TG_ERR_INVALID_ARGUMENT, TG_ERR_BAD_INPUT):
        raise ValueError(msg)
    if status == TG_ERR_NO_DEVICE:
        raise RuntimeError("No CUDA GPU found. " + msg)
    raise ToricLibError(status, msg)


def device_count() -> int:
    n = c_int32(0)
    check(load().tg_device_count(ctypes.byref(n)), "tg_device_count")
    return int(n.value)


def device_info(device: int) -> tuple[int, int, int, str]:
    sm, ma, mi = c_int32(0), c_int32(0), c_int32(0)
    name = ctypes.create_string_buffer(256)
    check(
        load().tg_device_info(
            device, ctypes.byref(sm), ctypes.byref(ma), ctypes.byref(mi), name, 256
        ),
        "tg_device_info",
    )
    return int(sm.value), int(ma.value), int(mi.value), name.value.decode()
