"""Build recipe of the CPU oracle: gcc -O2 -ffp-contract=off -fopenmp.

Produces oracle/lib/libcvlbm_oracle.so (git-ignored, travels with the tree).
"""

from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB = HERE / "lib" / "libcvlbm_oracle.so"
SRC = HERE / "cvlbm_oracle.c"
SRCS = (SRC, HERE / "char_stencil3d.c")
FLAGS = ["-O2", "-std=c11", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC", "-shared"]


def build(force: bool = False) -> Path:
    deps = [*SRCS, HERE / "cvlbm_oracle.h", HERE.parent / "include" / "cvlbm.h"]
    if not force and LIB.exists() and all(d.stat().st_mtime <= LIB.stat().st_mtime for d in deps):
        return LIB
    LIB.parent.mkdir(parents=True, exist_ok=True)
    tmp = LIB.with_suffix(".so.tmp")
    # the system gcc carries libgomp; other toolchains on PATH may not
    cands = [os.environ.get("CC"), "/usr/bin/gcc", shutil.which("gcc"), "cc"]
    last = None
    ccs = [c for c in cands if c]
    for flags in (FLAGS, [f for f in FLAGS if f != "-fopenmp"]):
        for cc in ccs:
            r = subprocess.run([cc, *flags, "-o", str(tmp), *map(str, SRCS), "-lm"], capture_output=True,
                               text=True)
            if r.returncode == 0:
                os.replace(tmp, LIB)
                return LIB
            last = r.stderr
    raise RuntimeError(f"oracle build failed: {last}")


if __name__ == "__main__":
    print(build(force=True))
