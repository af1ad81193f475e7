"""Generates tests/golden/golden.json from the reference's own Python code.

Run with the reference checkout given by --reference or the
TG_REFERENCE_DIR environment variable (one of them is required).  The reference modules import pyopencl/cupy at module level, so
both are stubbed; the functions used here are pure numpy/Python:
  gf8.MUL_TABLE                                 (gf8.py:24-38)
  precompute.build_eval_matrix                  (precompute.py:32-43)
  champion_search_canonical.precompute_gl2_perms, _rel_table,
      canonical_forms_batch (k <= 10), unpack_canonical  (:61-161)
max_zeros golden values come from a pure-Python brute force that follows the
reference's smoke test bf_max_zeros (kernel backup.py:203-222) over the
reference's own MUL_TABLE and M, plus the known answers of its smoke tests
(kernel backup.py:180-245).
"""

from __future__ import annotations

import argparse
import hashlib
import json
import os
import random
import sys
import types
from pathlib import Path

import numpy as np

OUT = Path(__file__).resolve().parent / "golden.json"


class _Stub(types.ModuleType):
    def __getattr__(self, name):
        return object


def brute_max_zeros(S, M, mul):
    k = len(S)
    best = 0
    rows = [M[s] for s in S]
    for pid in range(1, 8 ** k):
        acc = np.zeros(49, dtype=np.int64)
        for i in range(k):
            c = (pid >> (3 * i)) & 7
            if c:
                acc ^= mul[c][rows[i]]
        best = max(best, int((acc == 0).sum()))
    return best


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("TG_REFERENCE_DIR"),
                    help="reference checkout (default: $TG_REFERENCE_DIR)")
    args = ap.parse_args()
    if not args.reference:
        ap.error("give --reference or set TG_REFERENCE_DIR")
    sys.modules["pyopencl"] = _Stub("pyopencl")
    sys.modules["cupy"] = _Stub("cupy")
    sys.path.insert(0, args.reference)
    import champion_search_canonical as csc  # noqa: E402
    import gf8  # noqa: E402
    import precompute  # noqa: E402

    M = precompute.build_eval_matrix().astype(np.int32)
    mul = np.array(gf8.MUL_TABLE, dtype=np.int64)
    gl2 = csc.precompute_gl2_perms().astype(np.int32)
    rel = csc._rel_table().astype(np.uint8)

    rng = random.Random(20261203)
    # max_zeros known answers: the reference smoke tests + brute force.
    kat_sets = [[0], [0, 7], [0, 1, 7]]
    for _ in range(24):
        k = rng.randint(1, 4)
        kat_sets.append(sorted(rng.sample(range(49), k)))
    kats = [{"set": s, "max_zeros": brute_max_zeros(s, M, mul)} for s in kat_sets]

    # canonical keys by the reference's numpy path (k <= 10), grouped by k.
    canon = []
    for k in range(1, 11):
        sets = np.array([sorted(rng.sample(range(49), k)) for _ in range(30)], dtype=np.int32)
        keys = csc.canonical_forms_batch(sets, gl2)
        for row, key in zip(sets.tolist(), keys.tolist()):
            canon.append({"set": row, "key": int(key),
                          "unpacked": list(csc.unpack_canonical(int(key), k))})

    doc = {
        "generator": "tests/golden/make_golden.py",
        "mul_table": mul.tolist(),
        "eval_matrix": M.tolist(),
        "gl2_perms_sha256": hashlib.sha256(gl2.tobytes()).hexdigest(),
        "gl2_perms_rows": {"0": gl2[0].tolist(), "1000": gl2[1000].tolist(),
                           "2015": gl2[2015].tolist()},
        "rel_table_sha256": hashlib.sha256(rel.tobytes()).hexdigest(),
        "max_zeros_kats": kats,
        "smoke_known": {
            "S={0}": 0,
            "S={0,1,7}": 7,
            "abort_td49_fails": True,
            "exact_td42": 7,
        },
        "canonical_keys": canon,
        "canonical_orbit_counts": {"2": 1, "3": 3},
    }
    OUT.write_text(json.dumps(doc, separators=(",", ":")) + "\n")
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes)")


if __name__ == "__main__":
    main()
