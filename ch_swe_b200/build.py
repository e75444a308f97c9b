"""Build the sm_100a shared library ``ch_swe_b200/libchswe.so`` in-tree with nvcc."""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libchswe.so")
SOURCES = ["swe_api.cu"]
DEPS = ["swe_api.cu", "swe_common.cuh", "swe_kernels.cuh", "swe_tiled.cuh", "swe_sbp.cuh", "swe_advective.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build ch_swe_b200")


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, d) for d in DEPS] + [os.path.join(ROOT, "include", "chswe.h")]
    return all(os.path.getmtime(d) <= t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    # the device code is one large translation unit of templated kernels: let nvcc
    # optimise its kernels in parallel on the host's cores
    split = ["--split-compile", str(max(1, min(8, os.cpu_count() or 1)))]
    cmd = [nvcc(), "-O3", "-std=c++17", *ARCH, "-lineinfo", *split, "-Xcompiler", "-fPIC", "-shared",
           "-I", os.path.join(ROOT, "include"), "-I", CSRC, "-o", LIB + ".tmp",
           *[os.path.join(CSRC, s) for s in SOURCES]]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
