"""Build recipe for libwctb200.so (sm_100a, in-tree)."""

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libwctb200.so")
SOURCES = ["kernels.cu", "capi.cu", "pir.cpp"]
HEADERS = ["common.cuh", "fft.cuh", "kernels.cuh", "json.hpp", "pir.hpp"]

NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
    "--expt-relaxed-constexpr",
    "-shared",
]


def nvcc():
    for p in ("/usr/local/cuda/bin/nvcc", "nvcc"):
        if p == "nvcc" or os.path.exists(p):
            return p
    return "nvcc"


def stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    inc = os.path.join(os.path.dirname(HERE), "include", "wctb200.h")
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [inc, __file__]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=False):
    if not force and not stale():
        return LIB
    cmd = [nvcc()] + NVCC_FLAGS + [os.path.join(CSRC, s) for s in SOURCES] + ["-o", LIB + ".tmp"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True, cwd=CSRC)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force=True, verbose=True)
