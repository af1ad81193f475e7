"""Drop-in module with the name and API of the reference's kernel_canon.py
(`CanonicalOracle`, `init_canon_oracle`), served by the B200 canonical kernel."""

import sys
from pathlib import Path

_ROOT = str(Path(__file__).resolve().parents[2])
if _ROOT not in sys.path:
    sys.path.append(_ROOT)

from generalized_toric_gpu_search_b200.canonical import (  # noqa: E402,F401
    CanonicalOracle,
    init_canon_oracle,
)

__all__ = ["CanonicalOracle", "init_canon_oracle"]
