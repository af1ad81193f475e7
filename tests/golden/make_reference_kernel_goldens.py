"""Freezes the reference CUDA kernel's exact max_zeros at k = 12 and 13.

The reference kernel eval_min_distance_batch_bp (kernel_cuda_bp.py:146-238)
enumerates all 8^k - 1 messages of a set in one 256-thread block, so one
launch of 148 sets (one block per SM of a B200) takes about 40 s at k = 12
and about 6 minutes at k = 13 -- too long for a test, cheap enough to run
once.  This script runs it (oracle/_ref/libref_kernels.so, built from the
reference's own kernel source by oracle/build_ref.py, launched with the
reference wrapper's geometry) on seeded sets at target distance 1 (no early
exit) and writes the sets, the values and the launch times to a JSON fixture
that tests/test_reference_goldens_gpu.py compares the default path against.

Needs a B200 and the prebuilt oracle/_ref library:
  python tests/golden/make_reference_kernel_goldens.py --out FILE [--ks 12,13]
Sets: numpy default_rng(12000 + k), 148 sorted draws of k distinct indices
of 0..48 per k.
"""

from __future__ import annotations

import argparse
import ctypes
import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
REF_LIB = ROOT / "oracle" / "_ref" / "libref_kernels.so"
N = 49
N_SETS = 148


def seeded_sets(k: int, n: int = N_SETS) -> list[list[int]]:
    rng = np.random.default_rng(12000 + k)
    return [sorted(rng.choice(N, k, replace=False).tolist()) for _ in range(n)]


def main() -> None:
    import torch

    sys.path.insert(0, str(ROOT))
    from generalized_toric_gpu_search_b200.tables import build_eval_matrix

    ap = argparse.ArgumentParser()
    ap.add_argument("--out", type=Path, required=True)
    ap.add_argument("--ks", default="12,13")
    args = ap.parse_args()
    lib = ctypes.CDLL(str(REF_LIB))
    vp = ctypes.c_void_p
    lib.ref_bp_batch.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                 ctypes.c_longlong, ctypes.c_ulonglong, vp, vp]
    dev_M = torch.from_numpy(np.ascontiguousarray(build_eval_matrix().astype(np.int32))).cuda()
    doc = {"generator": "tests/golden/make_reference_kernel_goldens.py",
           "kernel": "eval_min_distance_batch_bp (kernel_cuda_bp.py:146-238), grid = sets, "
                     "block 256, target_distance 1",
           "device": torch.cuda.get_device_name(0), "by_k": {}}
    for k in [int(x) for x in args.ks.split(",")]:
        sets = seeded_sets(k)
        flat = torch.tensor([i for s in sets for i in s], dtype=torch.int32).cuda()
        out = torch.zeros(len(sets), dtype=torch.int32).cuda()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rc = lib.ref_bp_batch(dev_M.data_ptr(), flat.data_ptr(), k, N - 1, len(sets), 0, 0,
                              out.data_ptr(), None)
        if rc != 0:
            raise SystemExit(f"ref_bp_batch launch failed: {rc}")
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        doc["by_k"][str(k)] = {"seed": 12000 + k, "sets": sets, "max_zeros": out.cpu().tolist(),
                               "launch_seconds": dt,
                               "messages": float(len(sets) * (8 ** k - 1))}
        print(f"k={k}: {len(sets)} sets in {dt:.1f} s", flush=True)
        args.out.write_text(json.dumps(doc, separators=(",", ":")) + "\n")


if __name__ == "__main__":
    main()
