"""Builds the oracle (CPU restatement of the engine's march and of its world
producers) as oracle/liboracle.so.

Test infrastructure: only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg load the result.  Compiled without FMA contraction
(-ffp-contract=off) and without fast-math, so its float results follow the
same contract as the CUDA kernels.
"""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
LIB = HERE / "liboracle.so"
SRCS = [HERE / "vm_oracle.cpp", HERE / "producer.cpp", HERE / "atlas.cpp"]
DEPS = SRCS + [ROOT / "voxelcraft_menu_b200" / "csrc" / h for h in ("vm_types.h", "recipe.h")] + \
    [ROOT / "include" / "voxmarch_world.h"]


def build(force: bool = False) -> Path:
    if force or not LIB.exists() or any(d.stat().st_mtime > LIB.stat().st_mtime for d in DEPS):
        cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off", "-fno-fast-math",
               "-mno-fma", f"-I{ROOT}", *map(str, SRCS), "-o", str(LIB)]
        print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
