"""Drop-in module with the name of the reference's precompute.py: the same
tables (torus_points, bounding_cube_points, eval_monomial, build_eval_matrix)
and init_opencl / init_opencl_all with the reference's return shapes, handing
out B200 device handles instead of OpenCL objects.  The reference's drivers
import this module without pyopencl, and the oracles they build from its
handles (kernel.DistanceOracle here) run the sm_100a path."""

import sys
from pathlib import Path

_ROOT = str(Path(__file__).resolve().parents[2])
if _ROOT not in sys.path:
    sys.path.append(_ROOT)

from generalized_toric_gpu_search_b200.devices import (  # noqa: E402
    init_device as init_opencl,
    init_devices_all as init_opencl_all,
)
from generalized_toric_gpu_search_b200.tables import (  # noqa: E402
    bounding_cube_points,
    build_eval_matrix,
    eval_monomial,
    torus_points,
)

__all__ = ["torus_points", "bounding_cube_points", "eval_monomial", "build_eval_matrix",
           "init_opencl", "init_opencl_all"]
