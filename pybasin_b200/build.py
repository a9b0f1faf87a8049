"""In-tree build of the CUDA library ``pybasin_b200/_lib/libpybasin_b200.so``.

nvcc cross-compiles for sm_100a only (no GPU is needed to build).  Run
``python -m pybasin_b200.build`` or call :func:`build`.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT_DIR = PKG / "_lib"
LIB_NAME = "libpybasin_b200.so"
SOURCES = ["pb_api.cu", "pb_noalloc.cu", "pb_mlp.cu", "pb_order.cu", "pb_rtc.cu", "pb_mlp_tc.cu", "pb_train_tc.cu",
           "pb_train_fused.cu"]
ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build pybasin_b200")


def _inputs() -> list[Path]:
    files = [CSRC / s for s in SOURCES]
    files += sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + sorted((ROOT / "include").glob("*.h"))
    return files


def lib_path() -> Path:
    override = os.environ.get("PB_LIBRARY_PATH")
    return Path(override) if override else OUT_DIR / LIB_NAME


def is_stale() -> bool:
    out = lib_path()
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(p.stat().st_mtime > t for p in _inputs())


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile the library if it is missing or older than its sources."""
    out = lib_path()
    if not force and not is_stale():
        return out
    OUT_DIR.mkdir(parents=True, exist_ok=True)
    tmp = out.with_suffix(".so.tmp")
    cmd = [
        nvcc_path(),
        *ARCH_FLAGS,
        "-O3",
        "-lineinfo",
        "-std=c++17",
        *os.environ.get("PB_NVCC_DEFINES", "").split(),
        "-Xcompiler",
        "-fPIC",
        "-shared",
        "-I",
        str(ROOT / "include"),
        "-I",
        str(CSRC),
        "-o",
        str(tmp),
        *[str(CSRC / s) for s in SOURCES],
        "-ldl",
    ]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    tmp.replace(out)
    return out


if __name__ == "__main__":
    p = build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(p)
