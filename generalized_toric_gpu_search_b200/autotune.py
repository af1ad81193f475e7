"""Per-k launch-shape autotuner of the batched max_zeros kernels.

The information-set walk (the default enumeration for k >= 2) has three
knobs, tuned per k:
  is_blocks_per_sm     -- resident CTAs of 128 threads per SM (1..5);
  is_tasks_per_thread  -- a level is cut into about this many tasks per
                          resident thread (the equal-cost slice count);
  is_max_task_units    -- the largest task, in 49-codeword blocks (the slice
                          size cap; tasks align with supports).
The orbit walk (k = 1 by default, every k under TG_ENUM_ORBIT) has three:
  tail_rows R        -- one task covers the 8^R codewords of the last R rows;
  blocks_per_sm      -- resident CTAs per SM (register budget 128 or 64);
  threads_per_block  -- 64 / 128 / 256 threads per CTA.
Codes are not pinned to CTAs: every warp claims 32 tasks at a time from one
queue, so codes per CTA follow from the task size.  `tune` times every
candidate on a seeded calibration batch per k and records the fastest in a
JSON cache keyed by the GPU name; `ensure_table` tunes the information-set
knobs of the k it lacks (a few seconds), which DistanceOracleCUDABP does at
first use on a device without a table; `choose` returns the shape for a
batch by its largest k.
"""

from __future__ import annotations

import json
import os
import time
from pathlib import Path

import numpy as np

from .distance import LaunchConfig

CANDIDATES = [
    dict(tail_rows=r, blocks_per_sm=b, threads_per_block=t)
    for r in (3, 4, 5)
    for (b, t) in ((8, 128), (4, 128), (4, 256), (16, 64))
]

INFOSET_CANDIDATES = [
    dict(is_blocks_per_sm=b, is_tasks_per_thread=f, is_max_task_units=u)
    for b in (4, 5)
    for f in (4, 8, 16)
    for u in (49, 343, 2401)
]

INFOSET_KS = range(6, 16)
_SHAPE_KEYS = ("tail_rows", "blocks_per_sm", "threads_per_block", "is_blocks_per_sm",
               "is_tasks_per_thread", "is_max_task_units")


def cache_path() -> Path:
    root = os.environ.get("TORIC_B200_CACHE") or os.path.join(
        os.path.expanduser("~"), ".cache", "toric_b200")
    return Path(root) / "autotune.json"


def load_table(device_name: str, path: Path | None = None) -> dict[int, dict]:
    p = path or cache_path()
    if not p.exists():
        return {}
    try:
        doc = json.loads(p.read_text())
    except (OSError, ValueError):
        return {}
    return {int(k): v for k, v in doc.get(device_name, {}).items()}


def save_table(device_name: str, table: dict[int, dict], path: Path | None = None) -> Path:
    p = path or cache_path()
    p.parent.mkdir(parents=True, exist_ok=True)
    doc = {}
    if p.exists():
        try:
            doc = json.loads(p.read_text())
        except (OSError, ValueError):
            doc = {}
    doc[device_name] = {str(k): v for k, v in sorted(table.items())}
    # One temporary file per process: ranks of a multi-GPU run tune and save
    # at the same time, and each rename installs a complete file.
    tmp = p.with_suffix(f".{os.getpid()}.tmp")
    tmp.write_text(json.dumps(doc, indent=1, sort_keys=True))
    os.replace(tmp, p)
    return p


def choose(table: dict[int, dict], k_max: int) -> LaunchConfig | None:
    """Shape for a batch whose largest set has k_max rows: the entry of the
    nearest tuned k at or below k_max (work is dominated by the largest k);
    knobs an entry does not hold keep the library defaults."""
    if not table:
        return None
    ks = sorted(table)
    below = [k for k in ks if k <= k_max]
    k = below[-1] if below else ks[0]
    e = table[k]
    return LaunchConfig(**{key: int(e[key]) for key in _SHAPE_KEYS if key in e})


def calibration_sets(k: int, target_codewords: float = 2e10, seed: int = 97) -> list[list[int]]:
    """Seeded sets of size k whose orbit enumeration is ~target_codewords."""
    per_code = max(1.0, 0.2 * 8.0 ** max(k - 2, 1))
    n = int(min(4096, max(148, target_codewords / per_code)))
    rng = np.random.default_rng(seed + k)
    return [sorted(rng.choice(49, k, replace=False).tolist()) for _ in range(n)]


def infoset_calibration_sets(k: int, seed: int = 197) -> list[list[int]]:
    """Seeded sets of size k for the information-set walk (a few ms a batch)."""
    n = 4096 if k <= 9 else 1024
    rng = np.random.default_rng(seed + k)
    return [sorted(rng.choice(49, k, replace=False).tolist()) for _ in range(n)]


def measure(runner_factory, sets, config: LaunchConfig, reps: int = 2) -> float:
    """Best-of-reps seconds of one batched launch with `config`."""
    import torch

    from .distance import pack_sets

    runner = runner_factory(config)
    flat, off, kmax = pack_sets(sets)
    dev = runner.device
    d_idx, d_off = torch.from_numpy(flat).to(dev), torch.from_numpy(off).to(dev)
    d_out = torch.empty(len(sets), dtype=torch.int32, device=dev)
    p = runner.params(len(sets), kmax, 1)
    s = torch.cuda.current_stream(dev)
    runner.run(p, d_idx, d_off, d_out, stream=s)
    torch.cuda.synchronize(dev)
    best = float("inf")
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        runner.run(p, d_idx, d_off, d_out, stream=s)
        e1.record(s)
        torch.cuda.synchronize(dev)
        best = min(best, e0.elapsed_time(e1) / 1e3)
    return best


def tune(device_id: int = 0, ks=range(6, 16), candidates=None, path: Path | None = None,
         verbose: bool = False, walk: str = "orbit") -> dict[int, dict]:
    """Times every candidate shape per k and stores the fastest.  walk
    "orbit" tunes the orbit walk's knobs (enumeration TG_ENUM_ORBIT),
    "infoset" the information-set walk's (the default enumeration); the
    knobs of the other walk in a table entry are kept."""
    from . import _lib
    from .distance import DistanceRunner, ToricContext
    from .tables import build_eval_matrix

    infoset = walk == "infoset"
    cands = candidates or (INFOSET_CANDIDATES if infoset else CANDIDATES)
    ctx = ToricContext(device_id, build_eval_matrix())
    name = _lib.device_info(device_id)[3]
    table = load_table(name, path)
    for k in ks:
        sets = infoset_calibration_sets(k) if infoset else calibration_sets(k)
        results = []
        for c in cands:
            if c.get("tail_rows", 0) > k:
                continue
            cfg = LaunchConfig(**c) if infoset else \
                LaunchConfig(enumeration=2, **c)  # TG_ENUM_ORBIT: the walk these knobs shape
            t = measure(lambda cf: DistanceRunner(ctx, cf), sets, cfg)
            results.append((t, c))
            if verbose:
                print(f"[autotune] k={k:2d} {c} {1e3 * t:8.3f} ms")
        t_best, c_best = min(results, key=lambda x: x[0])
        entry = dict(table.get(k, {}))
        entry.update(c_best)
        entry["infoset_seconds" if infoset else "seconds"] = t_best
        entry["n_sets" if not infoset else "infoset_n_sets"] = len(sets)
        entry["tuned_at"] = time.strftime("%Y-%m-%dT%H:%M:%S")
        table[k] = entry
    save_table(name, table, path)
    ctx.close()
    return table


def ensure_table(device_id: int = 0, ks=INFOSET_KS, path: Path | None = None) -> dict[int, dict]:
    """The device's table, with the information-set knobs tuned for every k
    of ks that lacks them."""
    from . import _lib

    name = _lib.device_info(device_id)[3]
    table = load_table(name, path)
    missing = [k for k in ks if "is_tasks_per_thread" not in table.get(k, {})]
    if missing:
        table = tune(device_id, ks=missing, path=path, walk="infoset")
    return table
