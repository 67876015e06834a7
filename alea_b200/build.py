"""Build libalea_b200.so in-tree for sm_100a with nvcc.

    python -m alea_b200.build            # build if any source is newer
    python -m alea_b200.build --force
"""
from __future__ import annotations

import glob
import os
import re
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
    """True when the library is missing or older than an object's sources."""
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    for src in sources():
        obj = os.path.join(HERE, "_build", os.path.basename(src) + ".o")
        if not os.path.exists(obj) or os.path.getmtime(obj) > t:
            return True
        if any(os.path.getmtime(d) > os.path.getmtime(obj) for d in includes(src)):
            return True
    return False


def includes(path, seen=None):
    """The file and every quoted #include it reaches, recursively."""
    seen = set() if seen is None else seen
    path = os.path.normpath(path)
    if path in seen or not os.path.exists(path):
        return seen
    seen.add(path)
    for line in open(path, encoding="utf-8"):
        m = re.match(r'\s*#\s*include\s+"([^"]+)"', line)
        if m:
            includes(os.path.join(os.path.dirname(path), m.group(1)), seen)
    return seen


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile the sources whose object is older than the source or any header
    it includes, in parallel (the kernel files take minutes each), then link
    the shared library."""
    nvcc = os.environ.get("NVCC", "nvcc")
    obj_dir = os.path.join(HERE, "_build")
    os.makedirs(obj_dir, exist_ok=True)
    compile_flags = [f for f in NVCC_FLAGS if f != "-shared"]
    objs, jobs = [], []
    for src in sources():
        obj = os.path.join(obj_dir, os.path.basename(src) + ".o")
        objs.append(obj)
        stale = force or not os.path.exists(obj) or any(
            os.path.getmtime(d) > os.path.getmtime(obj) for d in includes(src))
        if not stale:
            continue
        cmd = [nvcc] + compile_flags + ["-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        jobs.append((obj, subprocess.Popen(cmd)))
    if not jobs and os.path.exists(LIB) and all(
            os.path.exists(o) and os.path.getmtime(o) <= os.path.getmtime(LIB) for o in objs):
        return LIB
    failed = [obj for obj, proc in jobs if proc.wait() != 0]
    if failed:
        for obj in failed:
            if os.path.exists(obj):
                os.remove(obj)
        raise subprocess.CalledProcessError(1, "nvcc -c " + " ".join(failed))
    cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB] + objs
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
