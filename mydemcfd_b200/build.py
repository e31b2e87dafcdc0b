"""Build recipe of the native library: nvcc for sm_100a, in-tree.

    python -m mydemcfd_b200.build        # -> mydemcfd_b200/libsmac_b200.so
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libsmac_b200.so")
SOURCES = [os.path.join(HERE, "csrc", "smac_api.cu"), os.path.join(HERE, "csrc", "smac_noalloc.cu"),
           os.path.join(HERE, "csrc", "smac_async.cu"), os.path.join(HERE, "csrc", "smac_post.cu"),
           os.path.join(HERE, "csrc", "smac_vti.cu")]
DEPS = SOURCES + [
    os.path.join(HERE, "csrc", "smac_common.cuh"),
    os.path.join(HERE, "csrc", "smac_kernels.cuh"),
    os.path.join(HERE, "csrc", "smac_rbgs.cuh"),
    os.path.join(HERE, "csrc", "smac_rbgs_tma.cuh"),
    os.path.join(HERE, "csrc", "smac_rbgs_zm.cuh"),
    os.path.join(HERE, "csrc", "smac_coarse_cluster.cuh"),
    os.path.join(ROOT, "include", "smac_b200.h"),
]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
]


def nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if os.path.exists(cand) else "nvcc"


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(p) > t for p in DEPS)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not stale():
        return LIB
    cmd = [nvcc(), *NVCC_FLAGS, "-I" + os.path.join(ROOT, "include"), "-o", LIB + ".tmp", *SOURCES]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
