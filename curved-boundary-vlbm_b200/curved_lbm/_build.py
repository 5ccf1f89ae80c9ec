"""Build recipe for libcvlbm.so (sm_100a) with nvcc.

The library is built in-tree, next to this file, so that the built object
travels with the source tree.  Parity builds use ``--fmad=false``: the kernels
then perform exactly the float64 operations of the reference solver.
"""

from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent
SRC_ROOT = PKG_DIR.parent  # curved-boundary-vlbm_b200/
REPO_ROOT = SRC_ROOT.parent
CSRC = SRC_ROOT / "csrc"
INCLUDE = REPO_ROOT / "include"
LIB_DIR = PKG_DIR / "_lib"
LIB_PATH = LIB_DIR / "libcvlbm.so"

SOURCES = ("cvlbm_api.cu", "cvlbm2d.cu", "cvlbm3d.cu", "cvlbm3d_geom.cu", "cvlbm_summary.cu",
           "cvlbm_gemm.cu",
           "cvlbm_fno.cu")
ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3",
    "-lineinfo",
    "--fmad=false",
    "-std=c++17",
    "-Xcompiler",
    "-fPIC",
    "-Xptxas",
    "-warn-spills",
]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libcvlbm.so")


def _stale() -> bool:
    if not LIB_PATH.exists():
        return True
    mtime = LIB_PATH.stat().st_mtime
    deps = [CSRC / s for s in SOURCES] + list(CSRC.glob("*.cuh")) + [INCLUDE / "cvlbm.h"]
    return any(d.stat().st_mtime > mtime for d in deps if d.exists())


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile every CUDA source into ``_lib/libcvlbm.so``; returns its path."""
    if not force and not _stale():
        return LIB_PATH
    LIB_DIR.mkdir(parents=True, exist_ok=True)
    nvcc = nvcc_path()
    objs = []
    for src in SOURCES:
        obj = LIB_DIR / (Path(src).stem + ".o")
        cmd = [nvcc, *ARCH_FLAGS, *NVCC_FLAGS, "-I", str(INCLUDE), "-c", str(CSRC / src), "-o",
               str(obj)]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        objs.append(str(obj))
    tmp = LIB_PATH.with_suffix(".so.tmp")
    cmd = [nvcc, *ARCH_FLAGS, "-shared", "-o", str(tmp), *objs, "-lcudart"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB_PATH)
    for o in objs:
        Path(o).unlink(missing_ok=True)
    return LIB_PATH


if __name__ == "__main__":
    print(build(force=True, verbose=True))
