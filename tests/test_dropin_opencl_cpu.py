"""The drop-in modules with the names of the reference's OpenCL-era modules
(dropin/precompute.py, dropin/kernel.py), on the CPU: the tables, the
initialisers' error without a GPU, DistanceOracle's signatures, handle checks
and size-limit messages (kernel.py:205-323, precompute.py:17-124), and, where
a reference checkout is present, that the reference's drivers import through
them without pyopencl."""

from __future__ import annotations

import importlib
import inspect
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest
import torch

from generalized_toric_gpu_search_b200 import devices, tables
from generalized_toric_gpu_search_b200.distance import DistanceOracleCUDABP

ROOT = Path(__file__).resolve().parents[1]
DROPIN = ROOT / "generalized_toric_gpu_search_b200" / "dropin"


@pytest.fixture(scope="module")
def mods():
    """precompute and kernel imported by the reference's module names."""
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


def test_tables_match_the_reference_definitions(mods):
    pre, _ = mods
    assert pre.torus_points() == [(x, y) for x in range(1, 8) for y in range(1, 8)]
    assert pre.bounding_cube_points() == [(a, b) for a in range(7) for b in range(7)]
    M = pre.build_eval_matrix()
    assert M.dtype == np.int32 and M.shape == (49, 49)
    want = np.array([[pre.eval_monomial(a, p) for p in pre.torus_points()]
                     for a in pre.bounding_cube_points()], dtype=np.int32)
    assert np.array_equal(M, want) and np.array_equal(M, tables.build_eval_matrix())
    assert pre.eval_monomial((0, 0), (5, 3)) == 1


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-GPU error")
def test_initialisers_raise_without_a_gpu(mods):
    pre, _ = mods
    for call in (pre.init_opencl, lambda: pre.init_opencl(allow_cpu=True), pre.init_opencl_all):
        with pytest.raises(RuntimeError, match="No CUDA GPU found"):
            call()


def test_signatures_bind_the_reference_call_sites(mods):
    _, ker = mods
    D = ker.DistanceOracle
    assert list(inspect.signature(D.__init__).parameters) == ["self", "ctx", "queue", "M_buf"]
    assert list(inspect.signature(D.max_zeros).parameters) == [
        "self", "s_indices", "target_distance"]
    sig = inspect.signature(D.max_zeros_batch)
    assert list(sig.parameters) == ["self", "batched_indices", "target_distance",
                                    "sample_count", "sample_seed"]
    assert sig.parameters["sample_count"].default == 0
    assert sig.parameters["sample_seed"].default == 0
    # champion_search.py:265-266 and evolve_search.py:205-206 shapes
    ctx = devices.DeviceContext(0, "x")
    q, buf = devices.DeviceQueue(ctx), devices.MatrixBuffer(ctx, tables.build_eval_matrix())
    inspect.signature(D).bind(ctx, q, buf)
    inspect.signature(D.max_zeros_batch).bind(None, [[0, 1]], 20, sample_count=5, sample_seed=3)


def test_handles_are_checked_before_any_device_work(mods):
    _, ker = mods
    M = tables.build_eval_matrix()
    c0, c1 = devices.DeviceContext(0), devices.DeviceContext(1)
    with pytest.raises(TypeError):
        ker.DistanceOracle(object(), object(), M)
    with pytest.raises(ValueError, match="different devices"):
        ker.DistanceOracle(c0, devices.DeviceQueue(c1), devices.MatrixBuffer(c0, M))
    with pytest.raises(ValueError, match="different devices"):
        ker.DistanceOracle(c0, devices.DeviceQueue(c0), devices.MatrixBuffer(c1, M))
    assert devices.DeviceQueue(c1).device == c1


def test_construction_reaches_the_b200_oracle(mods, monkeypatch):
    """With the B200 oracle's constructor replaced by a recorder, the handles
    pass their device index and matrix through."""
    _, ker = mods
    seen = []
    monkeypatch.setattr(DistanceOracleCUDABP, "__init__",
                        lambda self, device_id, M: seen.append((device_id, M)))
    M = tables.build_eval_matrix()
    ctx = devices.DeviceContext(1, "b200")
    q, buf = devices.DeviceQueue(ctx), devices.MatrixBuffer(ctx, M)
    o = ker.DistanceOracle(ctx, q, buf)
    assert seen == [(1, M)] and o.queue is q and o.M_buf is buf


def test_size_limits_raise_the_reference_messages(mods, monkeypatch):
    """kernel.py:246-247 and :288-291; within the limits the call goes to the
    B200 oracle's method."""
    _, ker = mods
    calls = []
    monkeypatch.setattr(DistanceOracleCUDABP, "max_zeros",
                        lambda self, s, td: calls.append(("one", len(s), td)) or 7)
    monkeypatch.setattr(DistanceOracleCUDABP, "max_zeros_batch",
                        lambda self, b, td, sc=0, ss=0: calls.append(("batch", len(b), sc)) or [])
    o = object.__new__(ker.DistanceOracle)
    with pytest.raises(ValueError, match="Exact OpenCL evaluation supports k <= 21"):
        o.max_zeros(list(range(22)), 10)
    assert o.max_zeros(list(range(21)), 10) == 7
    with pytest.raises(ValueError, match="OpenCL bit-parallel kernel supports k <= 49"):
        o.max_zeros_batch([list(range(49)) + [0]], 10, sample_count=100)
    with pytest.raises(ValueError, match="Exact OpenCL batch evaluation supports k <= 21"):
        o.max_zeros_batch([list(range(22))], 10)
    assert o.max_zeros_batch([list(range(30))], 10, sample_count=100, sample_seed=1) == []
    assert o.max_zeros_batch([], 10) == []
    assert calls == [("one", 21, 10), ("batch", 1, 100), ("batch", 0, 0)]


def _reference_dir() -> Path | None:
    sys.path.insert(0, str(ROOT))
    try:
        from oracle.build_ref import reference_dir
    finally:
        sys.path.remove(str(ROOT))
    d = reference_dir()
    return d if (d / "champion_search.py").is_file() else None


@pytest.mark.parametrize("driver", ["champion_search", "search", "evolve_search",
                                    "champion_search_canonical"])
def test_reference_drivers_import_through_the_dropin(driver):
    ref = _reference_dir()
    if ref is None:
        pytest.skip("no reference checkout")
    code = (
        "import sys, importlib\n"
        f"sys.path[:0] = [{str(DROPIN)!r}, {str(ref)!r}]\n"
        f"importlib.import_module({driver!r})\n"
        "import precompute, kernel\n"
        f"assert precompute.__file__.startswith({str(DROPIN)!r})\n"
        f"assert kernel.__file__.startswith({str(DROPIN)!r})\n"
        "assert 'pyopencl' not in sys.modules\n"
    )
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                         cwd=os.path.dirname(str(ref)), timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
