"""Build of the in-tree shared library libkaram_b200.so (sm_100a).

``python -m karam_b200.build`` compiles the CUDA kernels and the host C++
(topology analysis + C ABI) with nvcc into karam_b200/libkaram_b200.so. Only
symbols declared in include/karam.h are exported.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libkaram_b200.so")
SOURCES = ["kernels.cu", "topology.cpp", "abi.cpp", "noalloc.cu", "seeder.cu", "tc_gemm.cu", "spice.cpp"]
HEADERS = ["device.hpp", "topology.hpp", "nr_types.h", "nr_device.cuh", "noalloc.hpp", "seeder.hpp",
           "tc_gemm.hpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "karam.h"))
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps)


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    raise RuntimeError("nvcc not found")


def build(force=False, verbose=False):
    """Compiles libkaram_b200.so when a source is newer than the library."""
    if not force and not _stale():
        return LIB
    cmd = [nvcc(), "-O3", "-std=c++17", "-shared", "-lineinfo", *ARCH,
           "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
           "-Xptxas", "-v", "-I", os.path.join(ROOT, "include"),
           "-o", LIB + ".tmp", *[os.path.join(CSRC, f) for f in SOURCES]]
    res = subprocess.run(cmd, capture_output=True, text=True)
    log = os.path.join(HERE, "build.log")
    with open(log, "w") as fh:
        fh.write(" ".join(cmd) + "\n" + res.stdout + res.stderr)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed (see {log}):\n{res.stderr[-4000:]}")
    os.replace(LIB + ".tmp", LIB)
    if verbose:
        print(res.stderr)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
