"""The default path against frozen reference-kernel values at k = 12 and 13.

tests/golden/ref_kernel_k12_k13.json holds the exact max_zeros of 148 seeded
sets per k, computed once on a B200 by the reference's own CUDA kernel
(kernel_cuda_bp.py:146-238, built from its source) with
tests/golden/make_reference_kernel_goldens.py.  Those launches take about
40 s and 6 minutes, so the values are frozen rather than recomputed here.
"""

from __future__ import annotations

import json
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

FIXTURE = Path(__file__).resolve().parent / "golden" / "ref_kernel_k12_k13.json"
N = 49


def _goldens():
    return json.loads(FIXTURE.read_text())["by_k"]


@pytest.mark.parametrize("k", ["12", "13"])
def test_default_path_matches_frozen_reference(gpu_oracle, k):
    g = _goldens()[k]
    sets, want = g["sets"], g["max_zeros"]
    assert gpu_oracle.max_zeros_batch(sets, 1) == want
    # decisions at thresholds around the values
    for td in sorted({N - v for v in want})[:3]:
        tmax = N - td
        got = gpu_oracle.max_zeros_batch(sets, td)
        for e, a in zip(want, got):
            assert (a > tmax) == (e > tmax)
            if e <= tmax:
                assert a == e


@pytest.mark.parametrize("k", ["12", "13"])
def test_frozen_reference_values_have_witnesses(gpu_oracle, M, k):
    from oracle import oracle as orc

    g = _goldens()[k]
    values, wit = gpu_oracle.max_zeros_batch_witness(g["sets"], 1)
    assert values == g["max_zeros"]
    for s, v, w in zip(g["sets"], values, wit):
        assert orc.codeword_message(M, s, w)[0] == v


def test_k13_codes_stop_after_part_one_of_level_5(gpu_oracle):
    """After part 1 of level 5 (the supports holding the last row) a 13-row
    toric code's unseen codewords weigh at least ceil(49 * 5 / 12) = 21, so
    the codes with d <= 21 (most of the fixture) skip part 2; without the
    split every one of them would walk all C(12, 5) part-2 supports.  The
    stage counters add up to the walk's total."""
    from math import comb

    g = _goldens()["13"]
    assert gpu_oracle.max_zeros_batch(g["sets"], 1) == g["max_zeros"]
    runner = gpu_oracle._runner_for(13, False)
    stages = runner.stage_counters(gpu_oracle._stream)
    paths = runner.path_counters(gpu_oracle._stream)
    assert sum(stages.values()) == paths["infoset_codewords"]
    assert all(key == "1-3" or int(key.split(".")[0]) >= 4 for key in stages)
    part2 = comb(12, 5) * 7 ** 4
    n_high = sum(1 for v in g["max_zeros"] if N - v > 21)
    n_low = len(g["max_zeros"]) - n_high
    assert n_low > 100
    assert stages.get("5.1", 0) > 0
    assert stages.get("5.2", 0) <= (n_high + 5) * part2
