"""Drop-in module with the name and API of the reference's kernel_cuda_bp.py.

Put this directory first on sys.path and the reference drivers
(champion_search_canonical.py, evolve_search.py) import the B200 oracles
without a code change: `from kernel_cuda_bp import init_cuda_oracles_bp`.
"""

import sys
from pathlib import Path

_ROOT = str(Path(__file__).resolve().parents[2])
if _ROOT not in sys.path:
    sys.path.append(_ROOT)

from generalized_toric_gpu_search_b200.distance import (  # noqa: E402,F401
    DistanceOracleCUDABP,
    init_cuda_oracles_bp,
)

__all__ = ["DistanceOracleCUDABP", "init_cuda_oracles_bp"]
