"""Drop-in module with the name of the reference's kernel_cuda.py (the
fallback the drivers try when kernel_cuda_bp fails); it serves the same B200
oracles under the reference's older names."""

import sys
from pathlib import Path

_ROOT = str(Path(__file__).resolve().parents[2])
if _ROOT not in sys.path:
    sys.path.append(_ROOT)

from generalized_toric_gpu_search_b200.distance import (  # noqa: E402
    DistanceOracleCUDABP as DistanceOracleCUDA,
    init_cuda_oracles_bp as init_cuda_oracles,
)

__all__ = ["DistanceOracleCUDA", "init_cuda_oracles"]
