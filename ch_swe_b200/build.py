"""Build the sm_100a shared library ``ch_swe_b200/libchswe.so`` in-tree with nvcc."""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libchswe.so")
OBJDIR = os.path.join(HERE, "_build")
# the C ABI (edge sync, advective fluxes, quadrature, diagnostics) and one translation
# unit per precision and maximal tile for the stage and contravariant kernels: small
# device modules, compiled in parallel
STAGE_SOURCES = [f"stage_{p}{tm}.cu" for p in ("f", "d") for tm in (17, 25, 33)]
# the fused stage (TMA tiles, contravariant components in the stage) and its edge-strip
# kernel, one unit per precision
FUSED_SOURCES = ["fused_f.cu", "fused_d.cu"]
# the group launches (the RK4 stages of several contexts as one grid), one unit per
# precision
GROUP_SOURCES = ["group_f.cu", "group_d.cu"]
SOURCES = ["swe_api.cu", *STAGE_SOURCES, *FUSED_SOURCES, *GROUP_SOURCES]
COMMON_HEADERS = ["swe_common.cuh", "swe_kernels.cuh", "swe_sbp.cuh", "sbp63.h", "swe_advective.cuh", "swe_launch.cuh",
                  "swe_fused.cuh", "swe_tma.cuh"]
UNIT_HEADERS = {"swe_api.cu": COMMON_HEADERS + ["swe_ah.cuh", "swe_cgrid.cuh", "swe_diff.cuh", "lap63.h"],
                **{src: COMMON_HEADERS + ["fused_tu.cuh"] for src in FUSED_SOURCES}}
STAGE_HEADERS = COMMON_HEADERS + ["swe_tiled.cuh", "swe_stage_tu.cuh"]
UNIT_HEADERS.update({src: COMMON_HEADERS + ["swe_tiled.cuh", "swe_group.cuh", "group_tu.cuh"] for src in GROUP_SOURCES})
HEADERS = sorted(set(COMMON_HEADERS + UNIT_HEADERS["swe_api.cu"] + STAGE_HEADERS + ["fused_tu.cuh", "swe_group.cuh",
                                                                                    "group_tu.cuh"]))
DEPS = SOURCES + HEADERS
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


def _compile(src: str, verbose: bool, force: bool = False) -> str:
    obj = os.path.join(OBJDIR, os.path.splitext(src)[0] + ".o")
    deps = [os.path.join(CSRC, d) for d in [src, *UNIT_HEADERS.get(src, STAGE_HEADERS)]]
    if src == "swe_api.cu":   # the only unit that includes the C header
        deps.append(os.path.join(ROOT, "include", "chswe.h"))
    if not force and os.path.exists(obj) and all(os.path.getmtime(d) <= os.path.getmtime(obj) for d in deps):
        return obj
    cmd = [nvcc(), "-O3", "-std=c++17", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC", "-c",
           "-I", os.path.join(ROOT, "include"), "-I", CSRC, "-o", obj, os.path.join(CSRC, src)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(OBJDIR, exist_ok=True)
    jobs = max(1, min(len(SOURCES), os.cpu_count() or 1))
    # every unit is compiled whole: no --split-compile, whose partition of a unit's
    # kernels (and with it the generated code) varies from one run to the next
    with ThreadPoolExecutor(jobs) as pool:
        objs = list(pool.map(lambda src: _compile(src, verbose, force), SOURCES))
    subprocess.run([nvcc(), *ARCH, "-shared", "-o", LIB + ".tmp", *objs], check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
