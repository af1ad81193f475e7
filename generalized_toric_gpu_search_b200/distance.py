"""max_zeros oracles on the B200.

`DistanceOracleCUDABP` keeps the reference interface of
kernel_cuda_bp.py:246-323 (`device_id`, `max_zeros`, `max_zeros_batch` with
`sample_count` / `sample_seed`) and `init_cuda_oracles_bp` (:330-347), so the
search drivers (champion_search_canonical.py:611-647, evolve_search.py:190-220)
use it unchanged.  All arithmetic runs in libtoric_b200.so; torch only provides
device buffers and streams.

Result contract (the reference's, kernel_cuda_bp.py:227-235): a set passes when
max_zeros <= 49 - target_distance, and then the value is exact; a failing set
returns some witness > 49 - target_distance (the reference's value after an
early abort depends on thread timing, so only the decision is defined).
Sampled screening reproduces the reference's splitmix64 message multiset for
the same (set position, sample_seed), so a run without abort returns the same
maximum as the reference.
"""

from __future__ import annotations

import ctypes
import itertools
import threading
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from .tables import N_POINTS

MAX_EXACT_K = 21
MAX_SAMPLED_K = 49


@dataclass
class LaunchConfig:
    """Launch shape of the persistent distance kernel."""

    tail_rows: int = 0          # R; 0 = library default
    enumeration: int = _lib.TG_ENUM_AUTO
    variant: int = _lib.TG_VARIANT_AUTO
    blocks_per_sm: int = 0
    threads_per_block: int = 0
    # the information-set walk: CTAs per SM, tasks per resident thread of a
    # level, largest task in 49-codeword blocks (0 = library defaults 5, 4, 49)
    is_blocks_per_sm: int = 0
    is_tasks_per_thread: int = 0
    is_max_task_units: int = 0


def _require_cuda(device_id: int) -> None:
    if not torch.cuda.is_available() or _lib.device_count() == 0:
        raise RuntimeError("No CUDA GPU found.")
    if device_id < 0 or device_id >= torch.cuda.device_count():
        raise RuntimeError(f"CUDA device {device_id} does not exist")


class ToricContext:
    """One libtoric_b200 context (matrix tables on one device)."""

    def __init__(self, device_id: int, M: np.ndarray):
        _require_cuda(device_id)
        lib = _lib.load()
        m = np.ascontiguousarray(np.asarray(M, dtype=np.int32).reshape(N_POINTS, N_POINTS))
        handle = ctypes.c_void_p()
        _lib.check(
            lib.tg_context_create(
                device_id, m.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), ctypes.byref(handle)
            ),
            "tg_context_create",
        )
        self.handle = handle
        self.device_id = device_id
        flag = ctypes.c_int32(0)
        _lib.check(lib.tg_context_is_toric(handle, ctypes.byref(flag)), "tg_context_is_toric")
        self.is_toric = bool(flag.value)
        self.sm_count = _lib.device_info(device_id)[0]

    def close(self) -> None:
        if self.handle:
            _lib.load().tg_context_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass


def _load_packer():
    try:
        from . import _pack
    except ImportError:
        return None
    return _pack


_PACKER = _load_packer()


def pack_sets(batched_indices) -> tuple[np.ndarray, np.ndarray, int]:
    """Flattens a list of index lists into (flat int32, offsets int64, k_max).

    Sequences of Python ints go through the C packer (csrc/pack.c); other
    element types (floats, numpy arrays of them) through numpy.  An index
    that does not fit int32 comes back as -1, so a 0..48 range check on the
    flat array rejects it.
    """
    if _PACKER is not None:
        try:
            flat_b, off_b, k_max, _ = _PACKER.pack(batched_indices)
        except (TypeError, OverflowError):
            pass
        else:
            offsets = np.frombuffer(off_b, dtype=np.int64)
            flat = np.frombuffer(flat_b, dtype=np.int32, count=int(offsets[-1]))
            return flat, offsets, int(k_max)
    lengths = np.fromiter((len(s) for s in batched_indices), dtype=np.int64,
                          count=len(batched_indices))
    offsets = np.zeros(len(batched_indices) + 1, dtype=np.int64)
    np.cumsum(lengths, out=offsets[1:])
    flat = np.fromiter(itertools.chain.from_iterable(batched_indices), dtype=np.int32,
                       count=int(offsets[-1]))
    k_max = int(lengths.max()) if len(lengths) else 0
    return flat, offsets, k_max


class PinnedBatchStage:
    """Pinned host staging of packed batches, reused across calls.

    `pack` writes a batch straight into the pinned buffers with the C packer
    and returns (h_idx, h_off, k_max, bad) views of them, or None when the
    packer is missing or the items are not ints (the caller then packs with
    pack_sets).  After enqueueing the host-to-device copies out of the views,
    the caller calls `mark(stream)`; the next `pack` waits for those copies
    before it overwrites the buffers.  Not thread-safe: callers hold a lock.
    """

    def __init__(self):
        self.h_idx: torch.Tensor | None = None
        self.h_off: torch.Tensor | None = None
        self._copied: torch.cuda.Event | None = None

    def pack(self, batched_indices):
        if _PACKER is None or not hasattr(_PACKER, "pack_into"):
            return None
        n = len(batched_indices)
        if self._copied is not None:
            self._copied.synchronize()
        if self.h_off is None or self.h_off.numel() < n + 1:
            self.h_off = torch.empty(max(n + 1, 1 << 12), dtype=torch.int64, pin_memory=True)
        if self.h_idx is None:
            self.h_idx = torch.empty(1 << 16, dtype=torch.int32, pin_memory=True)
        for _ in range(2):
            try:
                total, k_max, bad, done = _PACKER.pack_into(
                    batched_indices, self.h_idx.data_ptr(), self.h_idx.numel(),
                    self.h_off.data_ptr(), self.h_off.numel())
            except (TypeError, OverflowError):
                return None
            if done:
                if total == 0:
                    self.h_idx[0] = 0
                return self.h_idx[:max(total, 1)], self.h_off[:n + 1], k_max, bad
            self.h_idx = torch.empty(max(total, 2 * self.h_idx.numel()), dtype=torch.int32,
                                     pin_memory=True)
        raise RuntimeError("batch packing did not fit its staging buffer")

    def pack_arrays(self, arrays):
        """The same for a list of int32 numpy arrays (numpy concatenation into
        the pinned buffers); returns (h_idx, h_off, k_max)."""
        n = len(arrays)
        lengths = np.fromiter((a.size for a in arrays), dtype=np.int64, count=n)
        total = int(lengths.sum())
        if self._copied is not None:
            self._copied.synchronize()
        if self.h_off is None or self.h_off.numel() < n + 1:
            self.h_off = torch.empty(max(n + 1, 1 << 12), dtype=torch.int64, pin_memory=True)
        if self.h_idx is None or self.h_idx.numel() < max(total, 1):
            self.h_idx = torch.empty(max(total, 1 << 16), dtype=torch.int32, pin_memory=True)
        off = self.h_off[:n + 1].numpy()
        off[0] = 0
        np.cumsum(lengths, out=off[1:])
        if total:
            np.concatenate(arrays, out=self.h_idx[:total].numpy())
        else:
            self.h_idx[0] = 0
        k_max = int(lengths.max()) if n else 0
        return self.h_idx[:max(total, 1)], self.h_off[:n + 1], k_max

    def mark(self, stream: torch.cuda.Stream) -> None:
        if self._copied is None:
            self._copied = torch.cuda.Event()
        self._copied.record(stream)


class DistanceRunner:
    """Device-level max_zeros: inputs and outputs are torch CUDA tensors.

    Owns a workspace that grows on demand and a CUDA stream; `run` enqueues
    the prep, scan and persistent walk kernels without synchronising.
    """

    def __init__(self, ctx: ToricContext, config: LaunchConfig | None = None):
        self.ctx = ctx
        self.config = config or LaunchConfig()
        self.device = torch.device("cuda", ctx.device_id)
        self._ws: torch.Tensor | None = None
        self.last_params: _lib.DistanceParams | None = None

    def params(self, n_sets: int, k_max: int, target_distance: int, sample_count: int = 0,
               sample_seed: int = 0) -> _lib.DistanceParams:
        c = self.config
        return _lib.DistanceParams(
            n_sets=n_sets, k_max=k_max, tail_rows=c.tail_rows, enumeration=c.enumeration,
            variant=c.variant, blocks_per_sm=c.blocks_per_sm,
            threads_per_block=c.threads_per_block, target_distance=int(target_distance),
            sample_count=int(sample_count), sample_seed=int(sample_seed) & (2**64 - 1),
            is_blocks_per_sm=c.is_blocks_per_sm, is_tasks_per_thread=c.is_tasks_per_thread,
            is_max_task_units=c.is_max_task_units,
        )

    def workspace(self, p: _lib.DistanceParams) -> torch.Tensor:
        need = ctypes.c_size_t(0)
        _lib.check(_lib.load().tg_distance_workspace_size(ctypes.byref(p), ctypes.byref(need)),
                   "tg_distance_workspace_size")
        if self._ws is None or self._ws.numel() < need.value:
            self._ws = torch.empty(max(int(need.value), 256), dtype=torch.uint8,
                                   device=self.device)
        return self._ws

    def run(self, p: _lib.DistanceParams, d_indices: torch.Tensor, d_offsets: torch.Tensor,
            d_out: torch.Tensor, d_target: torch.Tensor | None = None,
            d_set_ids: torch.Tensor | None = None, stream: torch.cuda.Stream | None = None,
            workspace: torch.Tensor | None = None) -> None:
        """Enqueues prepare + walk on `stream`."""
        self.prepare(p, d_indices, d_offsets, d_out, d_target, d_set_ids, stream, workspace)
        self.walk(p, d_out, stream, workspace)

    def prepare(self, p: _lib.DistanceParams, d_indices: torch.Tensor, d_offsets: torch.Tensor,
                d_out: torch.Tensor, d_target: torch.Tensor | None = None,
                d_set_ids: torch.Tensor | None = None, stream: torch.cuda.Stream | None = None,
                workspace: torch.Tensor | None = None) -> None:
        ws = workspace if workspace is not None else self.workspace(p)
        st = stream if stream is not None else torch.cuda.current_stream(self.device)
        self.last_params = p
        _lib.check(
            _lib.load().tg_max_zeros_prepare(
                self.ctx.handle, ctypes.byref(p), d_indices.data_ptr(), d_offsets.data_ptr(),
                d_target.data_ptr() if d_target is not None else None,
                d_set_ids.data_ptr() if d_set_ids is not None else None,
                d_out.data_ptr(), ws.data_ptr(), ws.numel(), st.cuda_stream,
            ),
            "tg_max_zeros_prepare",
        )

    def walk(self, p: _lib.DistanceParams, d_out: torch.Tensor,
             stream: torch.cuda.Stream | None = None,
             workspace: torch.Tensor | None = None,
             parts: int = _lib.TG_WALK_ENUMERATION | _lib.TG_WALK_INFOSET) -> None:
        """Enqueues the walks (`parts`: a mask of TG_WALK_* values)."""
        ws = workspace if workspace is not None else self.workspace(p)
        st = stream if stream is not None else torch.cuda.current_stream(self.device)
        _lib.check(
            _lib.load().tg_max_zeros_walk_part(self.ctx.handle, ctypes.byref(p), parts,
                                               d_out.data_ptr(), ws.data_ptr(), ws.numel(),
                                               st.cuda_stream),
            "tg_max_zeros_walk_part",
        )

    def run_witness(self, p: _lib.DistanceParams, d_indices: torch.Tensor,
                    d_offsets: torch.Tensor, d_out: torch.Tensor, d_witness: torch.Tensor,
                    d_target: torch.Tensor | None = None,
                    stream: torch.cuda.Stream | None = None) -> None:
        """Enqueues tg_max_zeros_witness: max_zeros into d_out and, per set, a
        codeword with exactly that many zeros into d_witness ((n, 49) uint8)."""
        st = stream if stream is not None else torch.cuda.current_stream(self.device)
        need = ctypes.c_size_t(0)
        _lib.check(_lib.load().tg_witness_workspace_size(ctypes.byref(p), ctypes.byref(need)),
                   "tg_witness_workspace_size")
        if self._ws is None or self._ws.numel() < need.value:
            self._ws = torch.empty(max(int(need.value), 256), dtype=torch.uint8,
                                   device=self.device)
        self.last_params = p
        _lib.check(
            _lib.load().tg_max_zeros_witness(
                self.ctx.handle, ctypes.byref(p), d_indices.data_ptr(), d_offsets.data_ptr(),
                d_target.data_ptr() if d_target is not None else None, None,
                d_out.data_ptr(), d_witness.data_ptr(), self._ws.data_ptr(), self._ws.numel(),
                st.cuda_stream,
            ),
            "tg_max_zeros_witness",
        )

    def status(self, p: _lib.DistanceParams, stream: torch.cuda.Stream) -> int:
        s = ctypes.c_int32(0)
        _lib.check(_lib.load().tg_distance_status(ctypes.byref(p), self._ws.data_ptr(),
                                                  stream.cuda_stream, ctypes.byref(s)),
                   "tg_distance_status")
        return int(s.value)

    def counters(self, stream: torch.cuda.Stream | None = None) -> tuple[int, int, float]:
        """(tasks, codewords evaluated, reference messages 8^k-1 summed) of the last run."""
        st = stream if stream is not None else torch.cuda.current_stream(self.device)
        t, c, r = ctypes.c_uint64(0), ctypes.c_uint64(0), ctypes.c_double(0.0)
        _lib.check(_lib.load().tg_distance_counters(ctypes.byref(self.last_params),
                                                    self._ws.data_ptr(), st.cuda_stream,
                                                    ctypes.byref(t), ctypes.byref(c),
                                                    ctypes.byref(r)),
                   "tg_distance_counters")
        return int(t.value), int(c.value), float(r.value)

    def path_counters(self, stream: torch.cuda.Stream | None = None) -> dict[str, int]:
        """Tasks and codewords of the last run, per walk."""
        st = stream if stream is not None else torch.cuda.current_stream(self.device)
        h = (ctypes.c_uint64 * 4)()
        _lib.check(_lib.load().tg_distance_path_counters(ctypes.byref(self.last_params),
                                                         self._ws.data_ptr(), st.cuda_stream, h),
                   "tg_distance_path_counters")
        return {"enumeration_tasks": int(h[0]), "enumeration_codewords": int(h[1]),
                "infoset_tasks_queued": int(h[2]), "infoset_codewords": int(h[3])}

    def stage_counters(self, stream: torch.cuda.Stream | None = None) -> dict[str, int]:
        """Codewords of the last run's information-set walk per stage: "1-3"
        (levels 1 to 3), then "w.1" and "w.2" for the two parts of level w
        (stages with no codeword are left out)."""
        st = stream if stream is not None else torch.cuda.current_stream(self.device)
        n = 2 * 21 + 2
        h = (ctypes.c_uint64 * n)()
        _lib.check(_lib.load().tg_distance_stage_counters(ctypes.byref(self.last_params),
                                                          self._ws.data_ptr(), st.cuda_stream,
                                                          h, n),
                   "tg_distance_stage_counters")
        out = {"1-3": int(h[0])} if h[0] else {}
        for i in range(1, n):
            if h[i]:
                out["%d.%d" % (i // 2, 2 if i % 2 else 1)] = int(h[i])
        return out


class DistanceOracleCUDABP:
    """Drop-in for the reference's DistanceOracleCUDABP (kernel_cuda_bp.py:246-323).

    `max_zeros_batch` also accepts sets of different sizes in one call (they
    share one persistent launch) and `target_distance` as a per-set sequence.
    """

    BLOCK_SIZE = 256  # kept for callers that read it; the B200 launch is persistent

    def __init__(self, device_id: int, M: np.ndarray, config: LaunchConfig | None = None,
                 autotune: bool = True):
        self.device_id = device_id
        self.ctx = ToricContext(device_id, M)
        self._fixed = config
        self._table: dict = {}
        if config is None and autotune:
            import os

            from .autotune import ensure_table, load_table

            # A device without a table is tuned at first use (a few seconds),
            # unless TORIC_B200_AUTOTUNE=0 asks for the library defaults.
            if os.environ.get("TORIC_B200_AUTOTUNE", "1") != "0":
                self._table = ensure_table(device_id)
            else:
                self._table = load_table(_lib.device_info(device_id)[3])
        self._runners: dict[tuple, DistanceRunner] = {}
        self.runner = self._runner_for(0, False)
        self.device = self.runner.device
        self._stream = torch.cuda.Stream(device=self.device)
        self._lock = threading.Lock()
        self._stage = PinnedBatchStage()

    def _runner_for(self, k_max: int, early_exit: bool) -> DistanceRunner:
        """Launch shape: the fixed config, else the autotuned one for k_max.
        The table is tuned on exact batches (every level walked); a sampled
        batch, or one whose thresholds can end sets early, keeps the library
        defaults, whose smaller tasks notice an early exit sooner."""
        cfg = self._fixed
        if cfg is None and not early_exit and self._table:
            from .autotune import choose

            cfg = choose(self._table, k_max)
        cfg = cfg or LaunchConfig()
        key = (cfg.tail_rows, cfg.enumeration, cfg.variant, cfg.blocks_per_sm,
               cfg.threads_per_block, cfg.is_blocks_per_sm, cfg.is_tasks_per_thread,
               cfg.is_max_task_units)
        r = self._runners.get(key)
        if r is None:
            r = self._runners[key] = DistanceRunner(self.ctx, cfg)
        return r

    # -- reference API --------------------------------------------------------

    def max_zeros(self, s_indices: list[int], target_distance: int) -> int:
        k = len(s_indices)
        if k == 0:
            return 0
        if k > MAX_EXACT_K:
            raise ValueError("Exact CUDA-BP evaluation supports k <= 21")
        return self._evaluate([list(s_indices)], target_distance, 0, 0)[0]

    def max_zeros_batch(self, batched_indices, target_distance, sample_count: int = 0,
                        sample_seed: int = 0) -> list[int]:
        num_sets = len(batched_indices)
        if num_sets == 0:
            return []
        return self._evaluate(batched_indices, target_distance, sample_count, sample_seed)

    def max_zeros_batch_witness(self, batched_indices, target_distance):
        """max_zeros_batch (exact) plus one witness codeword per set.

        Returns (values, witnesses): witnesses is an (n, 49) uint8 array of
        GF(8) symbols in M's column order, row s a codeword of set s's code
        with exactly values[s] zero coordinates (a minimum-weight codeword
        when the set passes, a codeword below the target distance when it
        fails; the zero codeword for dependent rows).  The reference returns
        only the counts; a caller can check a witness on the host by solving
        m M[S] = c."""
        n = len(batched_indices)
        if n == 0:
            return [], np.zeros((0, N_POINTS), dtype=np.uint8)
        flat, offsets, k_max = pack_sets(batched_indices)
        if k_max > MAX_EXACT_K:
            raise ValueError("Exact CUDA-BP batch evaluation supports k <= 21")
        if flat.size and (int(flat.min()) < 0 or int(flat.max()) >= N_POINTS):
            raise ValueError("exponent indices must lie in 0..48")
        per_set_td = not np.isscalar(target_distance)
        with self._lock, torch.cuda.device(self.device):
            s = self._stream
            with torch.cuda.stream(s):
                d_idx = torch.from_numpy(flat if flat.size else np.zeros(1, np.int32)).to(
                    self.device)
                d_off = torch.from_numpy(offsets).to(self.device)
                d_td = None
                if per_set_td:
                    td_arr = np.asarray(target_distance, dtype=np.int32)
                    if td_arr.shape != (n,):
                        raise ValueError("target_distance must be an int or one value per set")
                    d_td = torch.from_numpy(td_arr).to(self.device)
                d_out = torch.empty(n, dtype=torch.int32, device=self.device)
                d_wit = torch.empty((n, N_POINTS), dtype=torch.uint8, device=self.device)
                runner = self._runner_for(
                    k_max, not per_set_td and int(target_distance) > 1 or
                    per_set_td and bool((np.asarray(target_distance) > 1).any()))
                p = runner.params(n, k_max, 0 if per_set_td else int(target_distance))
                runner.run_witness(p, d_idx, d_off, d_out, d_wit, d_target=d_td, stream=s)
                h_out = d_out.to("cpu", non_blocking=True)
                h_wit = d_wit.to("cpu", non_blocking=True)
            status = runner.status(p, s)  # synchronises the stream
        if status != _lib.TG_OK:
            _lib.check(status, "max_zeros_batch_witness (device)")
        return h_out.numpy().tolist(), h_wit.numpy()

    def min_distance(self, s_indices: list[int], target_distance: int = 1) -> int:
        """49 - max_zeros (the helper of kernel backup.py:161-163)."""
        return N_POINTS - self.max_zeros(s_indices, target_distance)

    # -- implementation -------------------------------------------------------

    def _evaluate(self, batched_indices, target_distance, sample_count, sample_seed) -> list[int]:
        n = len(batched_indices)
        with self._lock, torch.cuda.device(self.device):
            staged = self._stage.pack(batched_indices)
            if staged is None:
                flat, offsets, k_max = pack_sets(batched_indices)
                bad = bool(flat.size) and (int(flat.min()) < 0 or int(flat.max()) >= N_POINTS)
                h_idx = torch.from_numpy(flat if flat.size else np.zeros(1, np.int32)).pin_memory()
                h_off = torch.from_numpy(offsets).pin_memory()
            else:
                h_idx, h_off, k_max, bad = staged
            if k_max > MAX_SAMPLED_K:
                raise ValueError("CUDA-BP bit-parallel kernel supports k <= 49")
            if sample_count <= 0 and k_max > MAX_EXACT_K:
                raise ValueError("Exact CUDA-BP batch evaluation supports k <= 21")
            if bad:
                raise ValueError("exponent indices must lie in 0..48")
            per_set_td = not np.isscalar(target_distance)
            td_arr = None
            if per_set_td:
                td_arr = np.asarray(target_distance, dtype=np.int32)
                if td_arr.shape != (n,):
                    raise ValueError("target_distance must be an int or one value per set")
            s = self._stream
            with torch.cuda.stream(s):
                d_idx = h_idx.to(self.device, non_blocking=True)
                d_off = h_off.to(self.device, non_blocking=True)
                self._stage.mark(s)
                d_td = None
                if td_arr is not None:
                    d_td = torch.from_numpy(td_arr).pin_memory().to(self.device, non_blocking=True)
                d_out = torch.empty(n, dtype=torch.int32, device=self.device)
                early = sample_count > 0 or (
                    bool((td_arr > 1).any()) if td_arr is not None else int(target_distance) > 1)
                self.runner = self._runner_for(k_max, early)
                p = self.runner.params(n, k_max, 0 if per_set_td else int(target_distance),
                                       sample_count if sample_count > 0 else 0, sample_seed)
                self.runner.run(p, d_idx, d_off, d_out, d_target=d_td, stream=s)
                h_out = torch.empty(n, dtype=torch.int32, pin_memory=True)
                h_out.copy_(d_out, non_blocking=True)
            status = self.runner.status(p, s)  # synchronises the stream
        if status != _lib.TG_OK:
            _lib.check(status, "max_zeros_batch (device)")
        return h_out.numpy().tolist()  # numpy converts faster than torch


def init_cuda_oracles_bp(M: np.ndarray) -> tuple[list[DistanceOracleCUDABP], int]:
    """One oracle per visible GPU and the SM count of device 0
    (kernel_cuda_bp.py:330-347)."""
    if not torch.cuda.is_available():
        raise RuntimeError("No CUDA GPU found.")
    n = _lib.device_count()
    if n == 0:
        raise RuntimeError("No CUDA GPU found.")
    oracles: list[DistanceOracleCUDABP] = []
    sm_count = 40
    for i in range(n):
        sm_i, _, _, name = _lib.device_info(i)
        print(f"[CUDA-B200] Device {i}: {name}  ({sm_i} SMs)")
        if i == 0:
            sm_count = sm_i
        oracles.append(DistanceOracleCUDABP(i, M))
    return oracles, sm_count


def dispatch_max_zeros_batch(oracles, batch, target_distance, sample_count: int = 0,
                             sample_seed: int = 0) -> list[int]:
    """A batch split over several oracles (one per GPU), as the reference's
    _dispatch does (champion_search_canonical.py:237-271): near-even contiguous
    chunks in device order, one host thread per device, and in sampled mode
    the seed of device i offset by i * 1_000_003 so each chunk reproduces the
    reference's per-device sampling.  Codes are independent, so there is no
    exchange between devices; results come back in batch order."""
    from concurrent.futures import ThreadPoolExecutor

    if not batch:
        return []
    n = len(oracles)

    def call(o, chunk, seed):
        if sample_count <= 0:
            return o.max_zeros_batch(chunk, target_distance)
        return o.max_zeros_batch(chunk, target_distance, sample_count=sample_count,
                                 sample_seed=seed)

    if n == 1:
        return call(oracles[0], batch, sample_seed)
    q, r = divmod(len(batch), n)
    chunks, start = [], 0
    for i in range(n):
        size = q + (1 if i < r else 0)
        chunks.append(batch[start:start + size])
        start += size
    with ThreadPoolExecutor(max_workers=n) as pool:
        futs = [pool.submit(call, o, c, sample_seed + i * 1_000_003)
                for i, (o, c) in enumerate(zip(oracles, chunks)) if c]
        out: list[int] = []
        for f in futs:
            out.extend(f.result())
    return out
