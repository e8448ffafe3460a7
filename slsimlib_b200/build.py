"""Build recipe of libglamer_b200.so (sm_100a) and of the oracle checker.

    python -m slsimlib_b200.build          # library only
    python -m slsimlib_b200.build --all    # + oracle/liboracle.so (+ oracle/_ref if the reference is present)
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libglamer_b200.so")
SOURCES = ["tree_build.cu", "rayshoot.cu", "field_plane.cu", "smoothing.cu"]
HEADERS = ["cosmology.h", "glb_internal.h", "glb_host.h", "halos.cuh", "walk.cuh", "walk_split.cuh", "walk_group.cuh", "walk_halos.cuh", "batch.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
    "--expt-relaxed-constexpr",
]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_library(force: bool = False, verbose: bool = False) -> str:
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "glamer_b200.h"))
    if not force and not _stale(LIB, deps):
        return LIB
    objs = []
    build_dir = os.path.join(HERE, "_build")
    os.makedirs(build_dir, exist_ok=True)
    for src in SOURCES:
        obj = os.path.join(build_dir, src.replace(".cu", ".o"))
        cmd = [nvcc(), *NVCC_FLAGS, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        subprocess.check_call(cmd)
        objs.append(obj)
    tmp = LIB + ".tmp"
    subprocess.check_call([nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", tmp, *objs,
                           "-lcudart"])
    os.replace(tmp, LIB)
    return LIB


def reference_dir():
    """The reference source tree the oracle binaries are compiled from (read
    only): $GLAMER_REFERENCE, else the checkout this build was prepared beside;
    None when neither exists (the GPU box: the binaries travel prebuilt)."""
    for d in (os.environ.get("GLAMER_REFERENCE"), "/root/reference"):
        if d and os.path.exists(os.path.join(d, "include", "quadTree.h")):
            return d
    return None


def build_oracle() -> None:
    cmd = ["make", "-s", "-C", os.path.join(ROOT, "oracle")]
    ref = reference_dir()
    if ref:
        cmd.append(f"REF={ref}")
    subprocess.check_call(cmd)


if __name__ == "__main__":
    build_library(force="--force" in sys.argv, verbose="-v" in sys.argv)
    if "--all" in sys.argv:
        build_oracle()
    print(LIB)
