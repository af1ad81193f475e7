"""Builds libtoric_b200.so (the sm_100a CUDA library) in-tree with nvcc.

Usage: python -m generalized_toric_gpu_search_b200.build [--ptxas-verbose]
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent
CSRC = PKG_DIR / "csrc"
LIB_NAME = "libtoric_b200.so"
LIB_PATH = PKG_DIR / LIB_NAME
SOURCES = ["abi.cu", "distance.cu", "canonical.cu", "intpeak.cu", "server.cu"]
ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libtoric_b200")
    return cand


def _newest_source_mtime() -> float:
    files = [CSRC / s for s in SOURCES] + list(CSRC.glob("*.cuh"))
    files.append(PKG_DIR.parent / "include" / "toric_b200.h")
    return max(f.stat().st_mtime for f in files if f.exists())


def needs_build() -> bool:
    return not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < _newest_source_mtime()


def build(force: bool = False, ptxas_verbose: bool = False) -> Path:
    """Compiles the CUDA sources into LIB_PATH (skipped when up to date)."""
    if not force and not ptxas_verbose and not needs_build():
        return LIB_PATH
    cmd = [
        nvcc_path(),
        *ARCH_FLAGS,
        "-O3",
        "-lineinfo",
        "-std=c++17",
        "--expt-relaxed-constexpr",
        "-Xcompiler",
        "-fPIC,-O2",
        "-shared",
        "-o",
        str(LIB_PATH) + f".{os.getpid()}.tmp",
        *[str(CSRC / s) for s in SOURCES],
    ]
    if ptxas_verbose:
        cmd.insert(1, "-Xptxas=-v")
    proc = subprocess.run(cmd, cwd=str(PKG_DIR), capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(
            "nvcc failed (exit %d):\n%s\n%s" % (proc.returncode, " ".join(cmd), proc.stderr)
        )
    if ptxas_verbose:
        sys.stderr.write(proc.stderr)
    # a per-process temporary name: ranks started together may build at once
    os.replace(str(LIB_PATH) + f".{os.getpid()}.tmp", LIB_PATH)
    return LIB_PATH


def pack_ext_path() -> Path:
    import sysconfig

    return PKG_DIR / ("_pack" + (sysconfig.get_config_var("EXT_SUFFIX") or ".so"))


def build_pack(force: bool = False) -> Path:
    """Compiles the host-side batch packer (csrc/pack.c, CPython C API) with
    the system C compiler (skipped when up to date)."""
    import sysconfig

    out = pack_ext_path()
    src = CSRC / "pack.c"
    if not force and out.exists() and out.stat().st_mtime >= src.stat().st_mtime:
        return out
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        raise RuntimeError("no C compiler found for the batch packer")
    cmd = [cc, "-O2", "-shared", "-fPIC", "-I" + sysconfig.get_paths()["include"], str(src),
           "-o", str(out) + f".{os.getpid()}.tmp"]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError("packer build failed:\n%s\n%s" % (" ".join(cmd), proc.stderr))
    os.replace(str(out) + f".{os.getpid()}.tmp", out)
    return out


if __name__ == "__main__":
    build(force=True, ptxas_verbose="--ptxas-verbose" in sys.argv)
    build_pack(force=True)
    print(LIB_PATH)
