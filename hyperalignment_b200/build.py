"""Builds the sm_100a shared library ``libha_b200.so`` in place (next to this file).

    python -m hyperalignment_b200.build

nvcc cross-compiles for sm_100a without a GPU.  The library links the CUDA
runtime statically and OpenMP (host-side accumulation) dynamically.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libha_b200.so")
SOURCES = [os.path.join(HERE, "csrc", "ha_b200.cu")]
DEPS = SOURCES + [os.path.join(HERE, "csrc", "ha_b200_kernels.cuh"), os.path.join(HERE, "csrc", "ha_b200_grid.cuh"), os.path.join(HERE, "csrc", "ha_b200_mlp.cuh"),
                  os.path.join(HERE, "csrc", "ha_b200_tc.cuh"), os.path.join(HERE, "csrc", "ha_b200_pca.cuh"),
                  os.path.join(ROOT, "include", "hyperalignment_b200.h")]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "-shared",
    "-Xcompiler", "-fPIC,-fopenmp,-O2",
    "-I" + os.path.join(ROOT, "include"),
]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(d) > t for d in DEPS)


def build(force: bool = False, verbose: bool = False, extra_flags=()) -> str:
    if force or needs_build():
        cmd = [nvcc(), *NVCC_FLAGS, *extra_flags, *SOURCES, "-o", LIB + ".tmp", "-lgomp"]
        if verbose:
            print(" ".join(cmd))
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            sys.stderr.write(res.stdout + res.stderr)
            raise RuntimeError("nvcc failed building libha_b200.so")
        if verbose and res.stderr:
            sys.stderr.write(res.stderr)
        os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    force = "--force" in sys.argv
    extra = ["-Xptxas", "-v"] if "--ptxas-v" in sys.argv else []
    print(build(force=force, verbose=True, extra_flags=extra))
