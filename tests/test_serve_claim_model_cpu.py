"""Host model of the served loop's task sizing and claim word
(srv_units / srv_task_units in csrc/serve_kernel.cuh, constants in
csrc/serve.cuh).

A request's stage st = 2 w + part - 1 is cut into tasks of nb units; warps
claim 32 tasks at a time with one atomicAdd on the claim word
id << 32 | st << 26 | next task.  A warp claims only while the task field
is below the stage's task count nt, but warps that checked at the same time
all add, so the field can pass nt by up to one claim per resident warp.  The
task size grows by factors of 7 until nt < kSrvMaxTasks, which leaves
2^26 - kSrvMaxTasks of headroom below the stage bits.  This test restates the
sizing and checks, for every k the loop accepts and every stage it can open,
that the tasks cover the stage, are aligned with supports, and that the
largest claim stays inside the task field.
"""

from __future__ import annotations

import re
from math import comb
from pathlib import Path

import pytest

CSRC = Path(__file__).resolve().parents[1] / "generalized_toric_gpu_search_b200" / "csrc"


def _const(name: str) -> int:
    for f in ("serve.cuh", "common.cuh"):
        m = re.search(rf"constexpr\s+[\w\s]+\b{name}\s*=\s*([^;]+);", (CSRC / f).read_text())
        if m:
            expr = m.group(1).split("//")[0].replace("ull", "")
            if "kMaxExactK" in expr:
                expr = expr.replace("kMaxExactK", str(_const("kMaxExactK")))
            return int(eval(expr, {}))  # shifts and sums of literals only
    raise KeyError(name)


TPB, PER_SM = _const("kSrvTPB"), _const("kSrvPerSm")
MAX_K, FIRST_STAGE = _const("kSrvMaxK"), _const("kSrvFirstStage")
TASK_MASK, MAX_TASKS = _const("kSrvTaskMask"), _const("kSrvMaxTasks")


def units_per_support(w: int) -> int:
    return 7 ** (w - 3) if w >= 3 else 1


def stage_units(k: int, st: int) -> int:
    """Supports of the stage (part 1: those holding row k - 1) x blocks."""
    w, part = st >> 1, (st & 1) + 1
    n_sup = comb(k - 1, w - 1) if part == 1 else comb(k - 1, w)
    return n_sup * units_per_support(w)


def task_units(units: int, w: int, lanes: int) -> int:
    target = 8 * lanes
    nb = max(1, min(-(-units // target), 343))
    bps = units_per_support(w)
    if bps > 1:
        if nb >= bps:
            nb = (nb // bps) * bps
        else:
            p7 = 1
            while p7 * 7 <= nb:
                p7 *= 7
            nb = 7 * p7 if nb * nb > 7 * p7 * p7 else p7
    while -(-units // nb) >= MAX_TASKS:
        nb *= 7
    return nb


def test_constants():
    assert TASK_MASK == (1 << 26) - 1 and 0 < MAX_TASKS < 1 << 26
    assert FIRST_STAGE == 2 * 4 + 1 - 1
    assert 2 * MAX_K + 2 - 1 < 64  # the stage field is 6 bits


@pytest.mark.parametrize("sms", [1, 148, 1024])
def test_every_stage_fits_the_claim_word(sms):
    lanes = sms * PER_SM * TPB
    warps = lanes // 32
    for k in range(4, MAX_K + 1):
        for w in range(4, k + 1):
            for part in (1, 2):
                st = 2 * w + part - 1
                units = stage_units(k, st)
                if units == 0:
                    continue
                nb = task_units(units, w, lanes)
                nt = -(-units // nb)
                bps = units_per_support(w)
                assert nt < MAX_TASKS and nt * nb >= units > (nt - 1) * nb
                assert nb % bps == 0 or bps % nb == 0  # whole supports, or a power of 7 in one
                # every resident warp past the check at once: one claim of 32 each
                assert (nt - 1) + 32 * warps + 32 <= TASK_MASK, (k, st, nt, lanes)


def test_tasks_beyond_343_blocks_stay_powers_of_7_and_fit_an_int():
    """Tasks grow past 343 blocks (the batch walk's largest) only where a
    stage would otherwise need more tasks than the field holds (high stages
    of k >= 15).  is_walk_blocks takes a task's blocks within one support as
    an int, and the tasks stay powers of 7 times 343."""
    lanes = 148 * PER_SM * TPB
    big = []
    for k in range(4, MAX_K + 1):
        for w in range(4, k + 1):
            for part in (1, 2):
                units = stage_units(k, 2 * w + part - 1)
                if units and task_units(units, w, lanes) > 343:
                    big.append((k, w, task_units(units, w, lanes)))
    assert big and min(k for k, _, _ in big) >= 15
    for _, w, nb in big:
        assert nb % 343 == 0
        q = nb // 343
        while q % 7 == 0:
            q //= 7
        assert q == 1 and min(nb, units_per_support(w)) < 2 ** 31
