"""Records the reference's own search drivers running against the drop-in API.

The drivers are imported unchanged from the reference checkout (cupy and
pyopencl stubbed: the modules only touch them inside the GPU classes):
  champion_search_canonical.canonical_champion_search   (:386-604), with its
      resume path load_canonical_state                   (:190-210)
  search.batched_bfs                                     (search.py:25-107)
  evolve_search.evaluate_sets                            (evolve_search.py:266-282)
They run with oracle objects that
  1. bind every call against this repository's drop-in signatures
     (DistanceOracleCUDABP.max_zeros_batch, init_canon_oracle, CanonicalOracle),
     so a call the drop-in would reject fails here, and
  2. answer on the CPU: canonical keys from the reference's own
     CPUCanonicalOracle (champion_search_canonical.py:143-150, numpy, k <= 10),
     max_zeros from the oracle (oracle/toric_oracle.c; exact, thresholded and
     splitmix64-sampled, the semantics of kernel_cuda_bp.py:146-238).
Every call with its answer, each level's (packed, sets, max_zeros) as
_pipelined_eval returned them, and the records the drivers wrote (or the
sha256 of the file) go to tests/golden/driver_traces.json.  Sets are stored
as 49-bit masks (bit i = exponent index i; every row the drivers pass is
sorted).  tests/test_driver_traces_cpu.py checks the host-side record writer
and resume reader against them; tests/test_dropin_replay_gpu.py replays the
calls through the drop-in modules on a B200 and checks every answer.

  python tests/golden/make_driver_traces.py --reference DIR   (or $TG_REFERENCE_DIR)
"""

from __future__ import annotations

import argparse
import contextlib
import hashlib
import importlib
import inspect
import json
import os
import sys
import tempfile
import types
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
OUT = Path(__file__).resolve().parent / "driver_traces.json"

# Target distances of the canonical searches (the role of codetables.de's
# bounds, which the drivers take as `targets`), chosen from the classes'
# distances (k = 2: 42; k = 3: 28, 35, 42; ...; k = 6: 14..36) so that every
# level has champions and failures.
TARGETS = {2: 42, 3: 42, 4: 40, 5: 36, 6: 35, 7: 34}


class _Stub(types.ModuleType):
    def __getattr__(self, name):
        if name.startswith("__"):
            raise AttributeError(name)
        return object


class Recorder:
    def __init__(self):
        self.calls: list[dict] = []

    def add(self, **rec):
        self.calls.append(rec)


def _sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def as_masks(rows) -> list[int]:
    """Sorted rows of distinct indices as 49-bit masks."""
    out = []
    for r in rows:
        r = [int(x) for x in r]
        if r != sorted(set(r)):
            raise AssertionError(f"row {r} is not sorted and distinct")
        out.append(sum(1 << x for x in r))
    return out


def make_fakes(rec: Recorder, M, csc):
    from generalized_toric_gpu_search_b200.canonical import CanonicalOracle, init_canon_oracle
    from generalized_toric_gpu_search_b200.distance import DistanceOracleCUDABP
    from oracle import oracle as orc

    sig_mzb = inspect.signature(DistanceOracleCUDABP.max_zeros_batch)
    sig_init = inspect.signature(init_canon_oracle)
    sig_canon = inspect.signature(CanonicalOracle.compute)

    class DistanceRecorder:
        """Stands in for DistanceOracleCUDABP(device_id, M)."""

        def __init__(self, device_id):
            self.device_id = device_id

        def max_zeros_batch(self, *args, **kwargs):
            b = sig_mzb.bind(self, *args, **kwargs)
            b.apply_defaults()
            a = b.arguments
            batch = [list(map(int, s)) for s in a["batched_indices"]]
            td, sc, seed = int(a["target_distance"]), int(a["sample_count"]), int(a["sample_seed"])
            out = orc.max_zeros_batch(M, batch, td, sample_count=sc, sample_seed=seed)
            rec.add(api="max_zeros_batch", device_id=self.device_id, sets=as_masks(batch),
                    target_distance=td, sample_count=sc, sample_seed=seed, result=out,
                    keywords=sorted(kwargs))
            return out

    class CanonRecorder:
        def __init__(self, gl2):
            self._cpu = csc.CPUCanonicalOracle(gl2)

        def compute(self, *args, **kwargs):
            b = sig_canon.bind(self, *args, **kwargs)
            sets = np.asarray(b.arguments["sets"])
            keys = [int(x) for x in self._cpu.compute(sets)]
            if keys != orc.canonical_keys(sets):
                raise AssertionError("oracle canonical keys differ from the reference's")
            rec.add(api="compute", k=int(sets.shape[1]), sets=as_masks(sets.tolist()),
                    result=keys)
            return np.array(keys, dtype=object)

    def fake_init_canon_oracle(*args, **kwargs):
        b = sig_init.bind(*args, **kwargs)
        a = b.arguments
        rec.add(api="init_canon_oracle", keywords=sorted(kwargs), positional=len(args),
                device_id=int(a["device_id"]),
                gl2_sha256=_sha(np.asarray(a["gl2_perms"], np.int32)),
                rel_sha256=_sha(np.asarray(a["rel_table"], np.uint8)))
        return CanonRecorder(np.asarray(a["gl2_perms"]))

    return DistanceRecorder, fake_init_canon_oracle


@contextlib.contextmanager
def in_dir(path: Path):
    old = os.getcwd()
    os.chdir(path)
    try:
        yield
    finally:
        os.chdir(old)


def read_jsonl(path: Path) -> list[dict]:
    return [json.loads(line) for line in path.read_text().splitlines() if line.strip()]


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("TG_REFERENCE_DIR"),
                    help="reference checkout (default: $TG_REFERENCE_DIR)")
    args = ap.parse_args()
    if not args.reference:
        ap.error("give --reference or set TG_REFERENCE_DIR")
    sys.path.insert(0, str(ROOT))
    import generalized_toric_gpu_search_b200.canonical  # noqa: F401  (torch before the stubs)
    sys.modules["pyopencl"] = _Stub("pyopencl")
    sys.modules["cupy"] = _Stub("cupy")
    sys.path.insert(1, args.reference)
    from oracle import oracle as orc

    orc.build()
    precompute = importlib.import_module("precompute")
    M = np.asarray(precompute.build_eval_matrix(), dtype=np.int32)
    lattice = precompute.bounding_cube_points()
    csc = importlib.import_module("champion_search_canonical")
    rec = Recorder()
    DistanceRecorder, fake_init = make_fakes(rec, M, csc)
    csc.init_canon_oracle = fake_init
    csc._HAS_GPU_CANON = True
    levels: list[dict] = []
    real_pipe = csc._pipelined_eval

    def recording_pipe(raw, canon_oracle, k, eval_distance, batch_size, oracles,
                       sample_count=0, sample_seed=0):
        packed, indices, mz = real_pipe(raw, canon_oracle, k, eval_distance, batch_size, oracles,
                                        sample_count=sample_count, sample_seed=sample_seed)
        levels.append({"k": k, "eval_distance": eval_distance, "batch_size": batch_size,
                       "sample_count": sample_count, "sample_seed": sample_seed,
                       "packed": [int(p) for p in packed], "sets": as_masks(indices),
                       "max_zeros": mz})
        return packed, indices, mz

    csc._pipelined_eval = recording_pipe
    doc: dict = {"generator": "tests/golden/make_driver_traces.py", "targets": TARGETS,
                 "scenarios": {}}

    def scenario(name: str, fn):
        rec.calls.clear()
        levels.clear()
        extra = fn() or {}
        doc["scenarios"][name] = {"calls": list(rec.calls), "levels": list(levels), **extra}
        print(f"{name}: {len(rec.calls)} calls, {len(levels)} levels", flush=True)

    with tempfile.TemporaryDirectory() as tmp:
        tmp = Path(tmp)

        def canonical_all():
            path = tmp / "canon_all.json"
            csc.canonical_champion_search(
                oracles=[DistanceRecorder(0)], lattice=lattice, results_file=path,
                targets=TARGETS, max_k=6, batch_size=500, prune_margin=None, resume=True,
                k_canonical_max=10, prune_eval_mode="champion")
            return {"config": {"max_k": 6, "batch_size": 500, "prune_margin": None,
                               "prune_eval_mode": "champion", "k_canonical_max": 10},
                    "records": read_jsonl(path)}

        def canonical_resume():
            path = tmp / "canon_resume.json"
            csc.canonical_champion_search(
                oracles=[DistanceRecorder(0)], lattice=lattice, results_file=path,
                targets=TARGETS, max_k=5, batch_size=500, prune_margin=None, resume=True)
            first = read_jsonl(path)
            last_k, survivors = csc.load_canonical_state(path)
            csc.canonical_champion_search(
                oracles=[DistanceRecorder(0)], lattice=lattice, results_file=path,
                targets=TARGETS, max_k=6, batch_size=500, prune_margin=None, resume=True)
            rec.calls.clear()  # the same calls as canonical_all's
            levels.clear()
            return {"config": {"max_k": [5, 6], "batch_size": 500, "prune_margin": None},
                    "records_first": first,
                    "file_sha256": hashlib.sha256(path.read_bytes()).hexdigest(),
                    "state_after_first": {"last_k": last_k, "survivors": sorted(survivors)}}

        def canonical_pruned_screened():
            path = tmp / "canon_pruned.json"
            csc.canonical_champion_search(
                oracles=[DistanceRecorder(0)], lattice=lattice, results_file=path,
                targets=TARGETS, max_k=6, batch_size=300, prune_margin=6, resume=False,
                k_canonical_max=10, prune_eval_mode="survivor", screen_from_k=5,
                screen_sample_count=3000, screen_seed=7, screen_candidate_log_limit=25)
            return {"config": {"max_k": 6, "batch_size": 300, "prune_margin": 6,
                               "prune_eval_mode": "survivor", "screen_from_k": 5,
                               "screen_sample_count": 3000, "screen_seed": 7,
                               "screen_candidate_log_limit": 25},
                    "records": read_jsonl(path)}

        def batched_bfs():
            search = importlib.import_module("search")
            with in_dir(tmp):
                search.batched_bfs(target_distance=42, oracle=DistanceRecorder(0),
                                   lattice=lattice, max_k=3)
                text = (tmp / "champions_batched.json").read_text()
            return {"config": {"target_distance": 42, "max_k": 3},
                    "n_records": len(json.loads(text)),
                    "file_sha256": hashlib.sha256(text.encode()).hexdigest()}

        def evaluate_sets():
            evo = importlib.import_module("evolve_search")
            rng = np.random.default_rng(4242)
            sets = [tuple(sorted(rng.choice(49, 12, replace=False).tolist())) for _ in range(64)]
            res = {}
            for td in (1, 24):
                res[str(td)] = evo.evaluate_sets([DistanceRecorder(0)], sets, td, 2048, 5, 16,
                                                 quiet=True)
            return {"config": {"sets": as_masks(sets), "sample_count": 2048,
                               "sample_seed": 5, "batch_size": 16}, "results": res}

        scenario("canonical_all", canonical_all)
        scenario("canonical_resume", canonical_resume)
        scenario("canonical_pruned_screened", canonical_pruned_screened)
        scenario("batched_bfs", batched_bfs)
        scenario("evaluate_sets", evaluate_sets)
    OUT.write_text(json.dumps(doc, separators=(",", ":")) + "\n")
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes)")


if __name__ == "__main__":
    main()
