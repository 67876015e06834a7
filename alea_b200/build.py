"""Build libalea_b200.so in-tree for sm_100a with nvcc.

    python -m alea_b200.build            # build if any source is newer
    python -m alea_b200.build --force
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libalea_b200.so")
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
]


def sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")) +
                  glob.glob(os.path.join(HERE, "csrc", "*.cpp")))


def deps():
    return (sources() + glob.glob(os.path.join(HERE, "csrc", "*.cuh")) +
            glob.glob(os.path.join(HERE, "csrc", "*.h")) +
            [os.path.join(ROOT, "include", "alea_gpu.h")])


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(p) > t for p in deps())


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc] + NVCC_FLAGS + ["-o", LIB] + sources()
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
