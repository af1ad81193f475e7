"""The reference's search drivers through the drop-in modules on a B200.

tests/golden/driver_traces.json holds every oracle call that the unchanged
reference drivers made -- canonical_champion_search
(champion_search_canonical.py:386-604) in three configurations,
search.batched_bfs (search.py:25-107) and evolve_search.evaluate_sets
(evolve_search.py:266-282) -- with their CPU answers.  Here the calls are
replayed, with the drivers' own arguments and keywords, through
generalized_toric_gpu_search_b200/dropin/ (imported under the reference's
module names kernel_cuda_bp and kernel_canon), so every answer the drivers
would get from the B200 is checked.  The device BFS (search.CanonicalBFS)
then runs the same canonical searches and must write the same records as
the reference driver, and resume the reference driver's partial file.
"""

from __future__ import annotations

import importlib
import json
import sys
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
DROPIN = ROOT / "generalized_toric_gpu_search_b200" / "dropin"
FIXTURE = ROOT / "tests" / "golden" / "driver_traces.json"
N = 49


def rows(masks):
    return [[i for i in range(N) if (int(m) >> i) & 1] for m in masks]


@pytest.fixture(scope="module")
def traces():
    return json.loads(FIXTURE.read_text())


@pytest.fixture(scope="module")
def dropin():
    """The drop-in modules imported by the reference's module names."""
    from generalized_toric_gpu_search_b200 import build as lib_build

    lib_build.build()
    saved = {m: sys.modules.pop(m, None) for m in ("kernel_cuda_bp", "kernel_canon")}
    sys.path.insert(0, str(DROPIN))
    try:
        bp = importlib.import_module("kernel_cuda_bp")
        canon = importlib.import_module("kernel_canon")
        assert Path(bp.__file__).parent == DROPIN and Path(canon.__file__).parent == DROPIN
        yield bp, canon
    finally:
        sys.path.remove(str(DROPIN))
        for m, v in saved.items():
            sys.modules.pop(m, None)
            if v is not None:
                sys.modules[m] = v


def _check_max_zeros(got, want, td):
    tmax = N - td
    for g, w in zip(got, want):
        assert (g > tmax) == (w > tmax)
        if w <= tmax:
            assert g == w


def test_replay_every_recorded_call(traces, dropin, M):
    from generalized_toric_gpu_search_b200.tables import precompute_gl2_perms, rel_table

    bp, canon_mod = dropin
    oracles, sm_count = bp.init_cuda_oracles_bp(M)
    assert sm_count > 0 and hasattr(oracles[0], "device_id")
    canon = None
    n_calls = 0
    tables = {"device_id": 0, "gl2_perms": precompute_gl2_perms(), "rel_table": rel_table()}
    for name, sc in traces["scenarios"].items():
        for c in sc["calls"]:
            n_calls += 1
            if c["api"] == "init_canon_oracle":
                canon = canon_mod.init_canon_oracle(**{kw: tables[kw] for kw in c["keywords"]})
            elif c["api"] == "compute":
                sets = np.array(rows(c["sets"]), dtype=np.int32).reshape(-1, c["k"])
                assert [int(x) for x in canon.compute(sets)] == c["result"], name
            elif c["api"] == "max_zeros_batch":
                o = oracles[c["device_id"]]
                batch = rows(c["sets"])
                if c["keywords"]:
                    got = o.max_zeros_batch(batch, c["target_distance"],
                                            sample_count=c["sample_count"],
                                            sample_seed=c["sample_seed"])
                elif c["sample_count"]:
                    got = o.max_zeros_batch(batch, c["target_distance"], c["sample_count"],
                                            c["sample_seed"])
                else:
                    got = o.max_zeros_batch(batch, c["target_distance"])
                if c["target_distance"] <= 1:
                    assert got == c["result"], name
                else:
                    _check_max_zeros(got, c["result"], c["target_distance"])
    assert n_calls > 30


@pytest.fixture(scope="module")
def opencl_dropin():
    """The drop-in precompute and kernel modules, imported by the reference's
    names (the OpenCL-era drivers' imports)."""
    from generalized_toric_gpu_search_b200 import build as lib_build

    lib_build.build()
    saved = {m: sys.modules.pop(m, None) for m in ("precompute", "kernel")}
    sys.path.insert(0, str(DROPIN))
    try:
        pre = importlib.import_module("precompute")
        ker = importlib.import_module("kernel")
        assert Path(pre.__file__).parent == DROPIN and Path(ker.__file__).parent == DROPIN
        yield pre, ker
    finally:
        sys.path.remove(str(DROPIN))
        for m, v in saved.items():
            sys.modules.pop(m, None)
            if v is not None:
                sys.modules[m] = v


def test_replay_through_the_opencl_era_names(traces, opencl_dropin):
    """The recorded max_zeros_batch calls through DistanceOracle(ctx, queue,
    M_buf) built from init_opencl(), as champion_search.py:265-266 builds it,
    and single-set max_zeros on the first sets of each exact call."""
    pre, ker = opencl_dropin
    ctx, queue, M_buf, M = pre.init_opencl()
    assert np.array_equal(M, pre.build_eval_matrix())
    o = ker.DistanceOracle(ctx, queue, M_buf)
    n_calls = 0
    for name, sc in traces["scenarios"].items():
        for c in sc["calls"]:
            if c["api"] != "max_zeros_batch" or c["device_id"] != 0:
                continue
            n_calls += 1
            batch = rows(c["sets"])
            td = c["target_distance"]
            got = o.max_zeros_batch(batch, td, c["sample_count"], c["sample_seed"])
            if td <= 1:
                assert got == c["result"], name
            else:
                _check_max_zeros(got, c["result"], td)
            if c["sample_count"] == 0:
                single = [o.max_zeros(s, td) for s in batch[:4]]
                _check_max_zeros(single, c["result"][:4], max(td, 1))
    assert n_calls > 10


def _by_kind(records):
    out: dict = {}
    for r in records:
        out.setdefault(r.get("type", "champion"), []).append(json.dumps(r, sort_keys=True))
    return {k: sorted(v) for k, v in out.items()}


def test_device_bfs_writes_the_reference_records(traces, tmp_path):
    """Unpruned canonical search to k = 6: the same classes, champions,
    survivors and level sentinels as the reference driver (order aside: the
    reference walks a Python set)."""
    from generalized_toric_gpu_search_b200.search import CanonicalBFS

    targets = {int(k): v for k, v in traces["targets"].items()}
    sc = traces["scenarios"]["canonical_all"]
    path = tmp_path / "canon.json"
    bfs = CanonicalBFS(0, dedup_capacity=1 << 16)
    levels = list(bfs.run(6, targets, None, results_file=path))
    assert [lv.k for lv in levels] == [2, 3, 4, 5, 6]
    got = [json.loads(x) for x in path.read_text().splitlines()]
    assert _by_kind(got) == _by_kind(sc["records"])


def test_device_bfs_pruned_survivor_mode(traces, tmp_path):
    """Survivor-mode pruning (evaluation at the keep distance): the exact
    levels match the reference driver record for record; the first screened
    level holds the same canonical classes (sampled values depend on each
    set's position in its batch, which follows the reference's Python set
    order)."""
    from generalized_toric_gpu_search_b200.search import CanonicalBFS

    targets = {int(k): v for k, v in traces["targets"].items()}
    sc = traces["scenarios"]["canonical_pruned_screened"]
    cfg = sc["config"]
    path = tmp_path / "canon.json"
    bfs = CanonicalBFS(0, dedup_capacity=1 << 16)
    list(bfs.run(cfg["max_k"], targets, cfg["prune_margin"],
                 prune_eval_mode=cfg["prune_eval_mode"], screen_from_k=cfg["screen_from_k"],
                 screen_sample_count=cfg["screen_sample_count"], screen_seed=cfg["screen_seed"],
                 batch_size=cfg["batch_size"],
                 screen_candidate_log_limit=cfg["screen_candidate_log_limit"],
                 results_file=path))
    got = [json.loads(x) for x in path.read_text().splitlines()]
    exact_k = cfg["screen_from_k"]
    assert _by_kind([r for r in got if r["k"] < exact_k]) == \
        _by_kind([r for r in sc["records"] if r["k"] < exact_k])
    first_screened = [lv for lv in sc["levels"] if lv["k"] == exact_k][0]
    ours = [r for r in got if r.get("type") == "level_complete" and r["k"] == exact_k][0]
    assert ours["n_canonical"] == len(first_screened["packed"])
    assert ours["screen_sample_count"] == cfg["screen_sample_count"] and not ours["verified"]


def test_device_bfs_resumes_the_reference_file(traces, tmp_path):
    """The reference driver's partial results file (levels up to 5) resumed
    by the device BFS: level 6 matches the uninterrupted reference run."""
    from generalized_toric_gpu_search_b200.search import CanonicalBFS, append_records

    targets = {int(k): v for k, v in traces["targets"].items()}
    res = traces["scenarios"]["canonical_resume"]
    path = tmp_path / "canon.json"
    append_records(res["records_first"], path)
    bfs = CanonicalBFS(0, dedup_capacity=1 << 16)
    levels = list(bfs.run(6, targets, None, results_file=path))
    assert [lv.k for lv in levels] == [6]
    got6 = [json.loads(x) for x in path.read_text().splitlines()][len(res["records_first"]):]
    want6 = [r for r in traces["scenarios"]["canonical_all"]["records"] if r["k"] == 6]
    assert _by_kind(got6) == _by_kind(want6)
