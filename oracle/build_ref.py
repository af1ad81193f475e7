"""ORACLE — test infrastructure only.  Recipe that builds the reference's own
CUDA kernels for the B200 from the reference sources, as a parity and speed
reference for the GPU tests.

The reference ships its kernels as CUDA C source strings inside Python
modules (kernel_cuda_bp.py `_CUDA_BP_SRC`, kernel_canon.py `_CUDA_CANON_SRC`)
that it compiles at run time with CuPy/NVRTC.  This script imports those two
modules from the reference checkout with `cupy` and `pyopencl` stubbed (the
modules only touch them inside methods), writes the two strings unchanged to
oracle/_ref/, and compiles them with nvcc for sm_100a together with
oracle/ref_harness.cu into oracle/_ref/libref_kernels.so.  oracle/_ref/ is
git-ignored (nothing of the reference is committed); a copy of the working tree
taken to a machine without the reference checkout carries the built library.

The reference checkout is taken from --reference, else from the
TG_REFERENCE_DIR environment variable, else from the recipe's fallback
location below (where the build container mounts it); build() does nothing
when none of them holds the reference.

Usage: python oracle/build_ref.py [--reference DIR]
"""

from __future__ import annotations

import argparse
import importlib
import os
import shutil
import subprocess
import sys
import types
from pathlib import Path

ORACLE_DIR = Path(__file__).resolve().parent
OUT_DIR = ORACLE_DIR / "_ref"
LIB = OUT_DIR / "libref_kernels.so"
FALLBACK_REFERENCE = Path("/root/reference")


def reference_dir() -> Path:
    """$TG_REFERENCE_DIR when set, else the fallback location."""
    env = os.environ.get("TG_REFERENCE_DIR")
    return Path(env) if env else FALLBACK_REFERENCE


class _Stub(types.ModuleType):
    def __getattr__(self, name):
        return object


def extract_sources(reference: Path) -> dict[str, str]:
    saved = {k: sys.modules.get(k) for k in ("cupy", "pyopencl", "kernel_cuda_bp",
                                             "kernel_canon")}
    sys.modules["cupy"] = _Stub("cupy")
    sys.modules["pyopencl"] = _Stub("pyopencl")
    sys.path.insert(0, str(reference))
    try:
        bp = importlib.import_module("kernel_cuda_bp")
        canon = importlib.import_module("kernel_canon")
        return {"ref_bp_src.cu": bp._CUDA_BP_SRC, "ref_canon_src.cu": canon._CUDA_CANON_SRC}
    finally:
        sys.path.remove(str(reference))
        for k, v in saved.items():
            if v is None:
                sys.modules.pop(k, None)
            else:
                sys.modules[k] = v


def build(reference: Path | None = None, force: bool = False) -> Path | None:
    """Builds oracle/_ref/libref_kernels.so; returns None when the reference
    checkout is absent (a machine without it uses the prebuilt library)."""
    reference = Path(reference) if reference is not None else reference_dir()
    if not (reference / "kernel_cuda_bp.py").exists():
        return LIB if LIB.exists() else None
    harness = ORACLE_DIR / "ref_harness.cu"
    if (not force and LIB.exists()
            and LIB.stat().st_mtime >= harness.stat().st_mtime
            and LIB.stat().st_mtime >= (reference / "kernel_cuda_bp.py").stat().st_mtime
            and LIB.stat().st_mtime >= (reference / "kernel_canon.py").stat().st_mtime):
        return LIB
    OUT_DIR.mkdir(exist_ok=True)
    for name, src in extract_sources(reference).items():
        (OUT_DIR / name).write_text(src)
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo",
           "-Xcompiler", "-fPIC", "-shared", "-I", str(ORACLE_DIR), "-o", str(LIB) + ".tmp",
           str(harness)]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError("reference kernel build failed:\n" + proc.stderr)
    Path(str(LIB) + ".tmp").replace(LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", type=Path, default=None,
                    help="reference checkout (default: $TG_REFERENCE_DIR, else the fallback)")
    ap.add_argument("--force", action="store_true")
    args = ap.parse_args()
    print(build(args.reference, args.force))
