"""B200-native GF(8) generalized-toric-code search hot path.

Drop-in oracle classes (same names and signatures as the reference modules
kernel_cuda_bp.py and kernel_canon.py) backed by libtoric_b200.so, the
hand-written sm_100a CUDA library:

  DistanceOracleCUDABP, init_cuda_oracles_bp   -- max_zeros / min distance
  CanonicalOracle, init_canon_oracle           -- AGL2(F7) canonical forms
  CanonicalDedup                               -- device hash-set dedup
  DistanceOracle, init_device, init_devices_all -- the same oracle with the
      signatures of the reference's OpenCL-era kernel.py / precompute.py

and the drivers built on them: ToricServer (device-resident request loop),
ToricServerPool (one loop per GPU), ToricBatchServer (micro-batches of the
batch path) and CanonicalBFS (the canonical search with every level on the
GPU).
"""

from .tables import (  # noqa: F401
    MUL_TABLE,
    N_POINTS,
    bounding_cube_points,
    build_eval_matrix,
    eval_monomial,
    gf8_mul,
    gf8_pow,
    indices_of,
    mask_of,
    pack_canonical,
    precompute_gl2_perms,
    rel_table,
    torus_points,
    unpack_canonical,
)

__all__ = [
    "DistanceOracleCUDABP",
    "init_cuda_oracles_bp",
    "CanonicalOracle",
    "init_canon_oracle",
    "CanonicalDedup",
    "DistanceOracle",
    "init_device",
    "init_devices_all",
    "LaunchConfig",
    "ToricServer",
    "ToricServerPool",
    "ToricBatchServer",
    "CanonicalBFS",
    "build_eval_matrix",
    "eval_monomial",
    "precompute_gl2_perms",
    "rel_table",
    "unpack_canonical",
]


def __getattr__(name):
    # The GPU classes import torch and the shared library lazily, so the host
    # tables stay importable on machines without either.
    if name in ("DistanceOracleCUDABP", "init_cuda_oracles_bp", "LaunchConfig",
                "DistanceRunner", "ToricContext", "pack_sets"):
        from . import distance

        return getattr(distance, name)
    if name in ("CanonicalOracle", "init_canon_oracle", "CanonicalDedup"):
        from . import canonical

        return getattr(canonical, name)
    if name in ("ToricServer", "ToricServerPool", "ToricBatchServer", "ServeAnswer"):
        from . import serve

        return getattr(serve, name)
    if name in ("DistanceOracle", "init_device", "init_devices_all"):
        from . import devices

        return getattr(devices, name)
    if name == "CanonicalBFS":
        from . import search

        return search.CanonicalBFS
    raise AttributeError(name)
