"""Drop-in module with the name of the reference's kernel.py, the OpenCL
oracle of the older drivers (champion_search.py, search.py, and the last
fallback of evolve_search.py): DistanceOracle(ctx, queue, M_buf), built from
the handles of the drop-in precompute.init_opencl / init_opencl_all, serves
the B200 path with the reference's methods and error messages."""

import sys
from pathlib import Path

_ROOT = str(Path(__file__).resolve().parents[2])
if _ROOT not in sys.path:
    sys.path.append(_ROOT)

from generalized_toric_gpu_search_b200.devices import DistanceOracle  # noqa: E402

__all__ = ["DistanceOracle"]
