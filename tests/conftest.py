"""pytest configuration: the `gpu` marker and import paths.

Tests marked `gpu` need a CUDA device (B200); everything else runs on CPU.
"""

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def golden():
    import json

    return json.loads((ROOT / "tests" / "golden" / "golden.json").read_text())


@pytest.fixture(scope="session")
def M():
    from generalized_toric_gpu_search_b200.tables import build_eval_matrix

    return build_eval_matrix()


def _has_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available() and torch.cuda.device_count() > 0
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu_oracle(M):
    if not _has_gpu():
        pytest.fail("gpu test collected without a CUDA device")
    from generalized_toric_gpu_search_b200 import build as _build
    from generalized_toric_gpu_search_b200.distance import DistanceOracleCUDABP

    _build.build()
    return DistanceOracleCUDABP(0, M)


@pytest.fixture(scope="session")
def canon_oracle():
    if not _has_gpu():
        pytest.fail("gpu test collected without a CUDA device")
    from generalized_toric_gpu_search_b200 import build as _build
    from generalized_toric_gpu_search_b200.canonical import CanonicalOracle

    _build.build()
    return CanonicalOracle(0)
