"""Device handles for callers written against the reference's OpenCL-era API
(precompute.py:66-124 init_opencl / init_opencl_all, kernel.py:205-323
DistanceOracle): one context per visible CUDA device, a queue on it and the
evaluation matrix bound to it.  The handles carry the device index and the
host matrix only; the oracle built from them is the B200
DistanceOracleCUDABP, so the older drivers (champion_search.py, search.py,
evolve_search.py's last fallback) run the same sm_100a path as the newer
ones.  There is no CPU device: without a CUDA GPU the initialisers raise, as
init_cuda_oracles_bp does.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .distance import DistanceOracleCUDABP
from .tables import build_eval_matrix


@dataclass(frozen=True)
class DeviceContext:
    """One CUDA device (the role of a cl.Context over one device)."""

    device_id: int
    name: str = ""


@dataclass(frozen=True)
class DeviceQueue:
    """A queue on a context (the role of a cl.CommandQueue); `device` is the
    context, as an OpenCL queue exposes its device."""

    context: DeviceContext

    @property
    def device(self) -> DeviceContext:
        return self.context


@dataclass(frozen=True, eq=False)
class MatrixBuffer:
    """The evaluation matrix bound to a context (the role of M_buf)."""

    context: DeviceContext
    host: np.ndarray


def _device_ids() -> list[int]:
    import torch

    from . import _lib

    if not torch.cuda.is_available():
        raise RuntimeError("No CUDA GPU found.")
    n = _lib.device_count()
    if n == 0:
        raise RuntimeError("No CUDA GPU found.")
    return list(range(n))


def init_devices_all() -> tuple[list[tuple[DeviceContext, DeviceQueue, MatrixBuffer]],
                                np.ndarray]:
    """([(ctx, queue, M_buf) per visible CUDA device], M), the return shape of
    the reference's init_opencl_all (precompute.py:66-82)."""
    from . import _lib

    ids = _device_ids()
    M = build_eval_matrix()
    out = []
    for i in ids:
        name = _lib.device_info(i)[3]
        ctx = DeviceContext(i, name)
        print(f"[precompute] CUDA device {i}: {name}")
        out.append((ctx, DeviceQueue(ctx), MatrixBuffer(ctx, M)))
    return out, M


def init_device(allow_cpu: bool = False) -> tuple[DeviceContext, DeviceQueue, MatrixBuffer,
                                                  np.ndarray]:
    """(ctx, queue, M_buf, M) on CUDA device 0, the return shape of the
    reference's init_opencl (precompute.py:85-124).  `allow_cpu` is accepted
    for that signature; there is no CPU path, so it changes nothing."""
    del allow_cpu
    triples, M = init_devices_all()
    ctx, queue, buf = triples[0]
    return ctx, queue, buf, M


class DistanceOracle(DistanceOracleCUDABP):
    """The reference's OpenCL DistanceOracle (kernel.py:205-323) on the B200
    path: built from the (ctx, queue, M_buf) that init_device /
    init_devices_all return, with the same max_zeros and max_zeros_batch and
    the same ValueError messages for the same size limits (kernel.py:246-247,
    :288-291).  Beyond those limits the methods are DistanceOracleCUDABP's:
    mixed k in one batch and per-set targets."""

    def __init__(self, ctx: DeviceContext, queue: DeviceQueue, M_buf: MatrixBuffer):
        if not (isinstance(ctx, DeviceContext) and isinstance(queue, DeviceQueue)
                and isinstance(M_buf, MatrixBuffer)):
            raise TypeError("DistanceOracle takes the (ctx, queue, M_buf) that the drop-in "
                            "precompute.init_opencl / init_opencl_all return")
        if queue.context != ctx or M_buf.context != ctx:
            raise ValueError("ctx, queue and M_buf belong to different devices")
        super().__init__(ctx.device_id, M_buf.host)
        self.queue = queue
        self.M_buf = M_buf

    def max_zeros(self, s_indices: list[int], target_distance: int) -> int:
        if len(s_indices) > 21:
            raise ValueError("Exact OpenCL evaluation supports k <= 21")
        return super().max_zeros(s_indices, target_distance)

    def max_zeros_batch(self, batched_indices: list[list[int]], target_distance: int,
                        sample_count: int = 0, sample_seed: int = 0) -> list[int]:
        if len(batched_indices) > 0:
            k = len(batched_indices[0])
            if k > 49:
                raise ValueError("OpenCL bit-parallel kernel supports k <= 49")
            if sample_count <= 0 and k > 21:
                raise ValueError("Exact OpenCL batch evaluation supports k <= 21")
        return super().max_zeros_batch(batched_indices, target_distance, sample_count,
                                       sample_seed)
