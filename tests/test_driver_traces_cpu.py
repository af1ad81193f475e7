"""The reference's search drivers, recorded against the drop-in API
(tests/golden/driver_traces.json, made by tests/golden/make_driver_traces.py
from the unchanged reference modules), checked on the host:

  * every recorded call binds to this repository's drop-in signatures, and
    its answer is the oracle's (the canonical keys were produced by the
    reference's own numpy path);
  * level_records reproduces canonical_champion_search's JSONL records
    (champion_search_canonical.py:531-583) from the same level data, and the
    reference's resumed results file byte for byte;
  * load_canonical_state reads the reference's partial file as the
    reference's resume does (:190-210).
"""

from __future__ import annotations

import hashlib
import inspect
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as orc

FIXTURE = Path(__file__).resolve().parent / "golden" / "driver_traces.json"


@pytest.fixture(scope="module")
def traces():
    return json.loads(FIXTURE.read_text())


def rows(masks):
    return [[i for i in range(49) if (int(m) >> i) & 1] for m in masks]


def test_recorded_calls_bind_to_dropin_signatures(traces):
    from generalized_toric_gpu_search_b200.canonical import init_canon_oracle
    from generalized_toric_gpu_search_b200.distance import DistanceOracleCUDABP

    init_sig = inspect.signature(init_canon_oracle)
    mzb_sig = inspect.signature(DistanceOracleCUDABP.max_zeros_batch)
    seen = set()
    for sc in traces["scenarios"].values():
        for c in sc["calls"]:
            if c["api"] == "init_canon_oracle":
                # the reference driver passes device_id, gl2_perms, rel_table by keyword
                init_sig.bind(**{kw: None for kw in c["keywords"]})
                seen.add(tuple(c["keywords"]))
            elif c["api"] == "max_zeros_batch" and c["keywords"]:
                mzb_sig.bind(None, [], 1, **{kw: 0 for kw in c["keywords"]})
    assert ("device_id", "gl2_perms", "rel_table") in seen


def test_recorded_answers_are_the_oracles(traces, M):
    for name, sc in traces["scenarios"].items():
        for c in sc["calls"]:
            if c["api"] == "compute":
                sets = np.array(rows(c["sets"]), dtype=np.int32).reshape(-1, c["k"])
                assert orc.canonical_keys(sets) == c["result"], name
            elif c["api"] == "max_zeros_batch":
                got = orc.max_zeros_batch(M, rows(c["sets"]), c["target_distance"],
                                          sample_count=c["sample_count"],
                                          sample_seed=c["sample_seed"])
                assert got == c["result"], name


def _replay_levels(sc, targets):
    from generalized_toric_gpu_search_b200.search import level_records
    from generalized_toric_gpu_search_b200.tables import bounding_cube_points

    cfg = sc["config"]
    lattice = bounding_cube_points()
    out = []
    for lv in sc["levels"]:
        k = lv["k"]
        recs, _ = level_records(
            k, lv["packed"], rows(lv["sets"]), lv["max_zeros"], lattice, targets.get(k, 1),
            prune_margin=cfg.get("prune_margin"),
            prune_eval_mode=cfg.get("prune_eval_mode", "champion"),
            sample_count=lv["sample_count"],
            screen_candidate_log_limit=cfg.get("screen_candidate_log_limit", 200))
        out.extend(recs)
    return out


@pytest.mark.parametrize("name", ["canonical_all", "canonical_pruned_screened"])
def test_level_records_reproduce_reference_records(traces, name):
    targets = {int(k): v for k, v in traces["targets"].items()}
    sc = traces["scenarios"][name]
    got = _replay_levels(sc, targets)
    assert got == sc["records"]
    assert [json.dumps(r) for r in got] == [json.dumps(r) for r in sc["records"]]
    kinds = {r.get("type", "champion") for r in got}
    assert {"survivor", "level_complete", "champion"} <= kinds
    if name == "canonical_pruned_screened":
        assert "candidate" in kinds


def test_resume_state_and_resumed_file(traces, tmp_path):
    from generalized_toric_gpu_search_b200.search import (append_records, level_records,
                                                          load_canonical_state)
    from generalized_toric_gpu_search_b200.tables import bounding_cube_points

    targets = {int(k): v for k, v in traces["targets"].items()}
    res = traces["scenarios"]["canonical_resume"]
    path = tmp_path / "canon.json"
    assert load_canonical_state(path) == (1, {0})
    append_records(res["records_first"], path)
    last_k, surv = load_canonical_state(path)
    assert last_k == res["state_after_first"]["last_k"]
    assert sorted(surv) == res["state_after_first"]["survivors"]
    # the resumed run appends level 6, whose data the uninterrupted run recorded
    lv6 = [lv for lv in traces["scenarios"]["canonical_all"]["levels"] if lv["k"] == 6][0]
    recs, _ = level_records(6, lv6["packed"], rows(lv6["sets"]), lv6["max_zeros"],
                            bounding_cube_points(), targets[6])
    append_records(recs, path)
    assert hashlib.sha256(path.read_bytes()).hexdigest() == res["file_sha256"]


def test_batched_bfs_file_from_recorded_answers(traces):
    """search.batched_bfs's champions file (search.py:63-104) follows from the
    recorded answers; checks that the recorded calls are the ones it made."""
    from generalized_toric_gpu_search_b200.tables import bounding_cube_points

    sc = traces["scenarios"]["batched_bfs"]
    td = sc["config"]["target_distance"]
    lattice = bounding_cube_points()
    results = []
    for c in sc["calls"]:
        k = len(rows(c["sets"][:1])[0])
        for s, mz in zip(rows(c["sets"]), c["result"]):
            if mz <= 49 - td:
                results.append({"indices": s, "lattice_points": [list(lattice[i]) for i in s],
                                "k": k, "max_zeros": mz, "min_distance": 49 - mz,
                                "target_distance": td})
    text = json.dumps(results, indent=2)
    assert hashlib.sha256(text.encode()).hexdigest() == sc["file_sha256"]
