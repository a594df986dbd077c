"""Builds the in-tree shared library of the march (libvoxmarch.so) for sm_100a.

nvcc cross-compiles without a GPU, so this runs on any machine with CUDA 12.9.
The CUDA translation units are compiled with --fmad=false and IEEE division /
square root: the traversal's float arithmetic must not be contracted, so that
voxel, face and t agree bit for bit with the CPU restatement of the engine's
WGSL march.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
ROOT = PKG.parent
BUILD = PKG / "_build"
LIB = PKG / "libvoxmarch.so"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "--fmad=false", "-prec-div=true", "-prec-sqrt=true",
    "-ftz=false", "-Xcompiler", "-fPIC", "-Xcompiler", "-fopenmp", f"-I{ROOT}", f"-I{CSRC}",
]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-fopenmp", "-ffp-contract=off", f"-I{ROOT}", f"-I{CSRC}"]

CU_SOURCES = ["kernels.cu", "pipeline.cu", "capi.cu", "gbuffer.cu", "shade.cu", "static_scratch.cu", "soften.cu",
              "encode.cu", "resolve.cu"]
# The shading model is held to tolerances against FP64, not to bit equality
# with the oracle, so it may contract a * b + c into fused multiply-adds.
CU_EXTRA = {"shade.cu": ["--fmad=true"]}
CPP_SOURCES = ["store.cpp", "look.cpp"]
HEADERS = ["vm_types.h", "march_device.cuh", "kernels.cuh", "ray_stages.cuh", "shade.cuh", "store.h", "recipe.h",
           "water.cuh", "resolve.cuh"]


def _newer(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str]) -> None:
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(verbose_ptxas: bool = False, force: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    headers = [CSRC / h for h in HEADERS] + [ROOT / "include" / "voxmarch.h", ROOT / "include" / "voxmarch_world.h"]
    objs = []
    for src in CU_SOURCES:
        obj = BUILD / (src + ".o")
        if force or verbose_ptxas or _newer(obj, [CSRC / src] + headers):
            extra = ["-Xptxas", "-v"] if verbose_ptxas else []
            own = CU_EXTRA.get(src, [])
            flags = [f for f in NVCC_FLAGS if not any(f.split("=")[0] == o.split("=")[0] for o in own)]
            _run([NVCC, *flags, *own, *extra, "-c", str(CSRC / src), "-o", str(obj)])
        objs.append(obj)
    for src in CPP_SOURCES:
        obj = BUILD / (src + ".o")
        if force or _newer(obj, [CSRC / src] + headers):
            _run(["g++", *CXX_FLAGS, "-c", str(CSRC / src), "-o", str(obj)])
        objs.append(obj)
    if force or _newer(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-Xcompiler", "-fopenmp", "-lgomp",
              "-lcudart"])
    return LIB


if __name__ == "__main__":
    build(verbose_ptxas="-v" in sys.argv, force="--force" in sys.argv)
