"""Build recipe for libwctb200.so (sm_100a, in-tree)."""

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libwctb200.so")
SOURCES = ["kernels.cu", "adjoint.cu", "dft.cu", "splat.cu", "capi.cu", "pir.cpp"]
HEADERS = ["common.cuh", "fft.cuh", "gauss.cuh", "kernels.cuh", "rng.cuh", "fft_lengths.h", "json.hpp", "pir.hpp"]

NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
    "--expt-relaxed-constexpr",
    "-shared", "-Xlinker", "-soname=libwctb200.so",
]

AUTOGRAD_SRC = os.path.join(CSRC, "autograd.cpp")
AUTOGRAD_NAME = "_wct_autograd"


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


def autograd_path():
    import sysconfig
    return os.path.join(HERE, AUTOGRAD_NAME + sysconfig.get_config_var("EXT_SUFFIX"))


def autograd_stale():
    out = autograd_path()
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    inc = os.path.join(os.path.dirname(HERE), "include", "wctb200.h")
    return any(os.path.getmtime(d) > t for d in (AUTOGRAD_SRC, inc, __file__, LIB) if os.path.exists(d))


def build_autograd(force=False, verbose=False):
    """The libtorch autograd extension (host C++ only; links libwctb200.so)."""
    out = autograd_path()
    if not force and not autograd_stale():
        return out
    import sysconfig
    import torch
    from torch.utils import cpp_extension as ce
    build(force=False)
    incs = ce.include_paths(device_type="cuda")
    libs = ce.library_paths(device_type="cuda")
    abi = int(torch._C._GLIBCXX_USE_CXX11_ABI)
    cmd = ["g++", "-O2", "-std=c++17", "-shared", "-fPIC", AUTOGRAD_SRC, "-o", out + ".tmp",
           "-DTORCH_EXTENSION_NAME=" + AUTOGRAD_NAME, "-DTORCH_API_INCLUDE_EXTENSION_H",
           "-D_GLIBCXX_USE_CXX11_ABI=%d" % abi, "-I" + sysconfig.get_paths()["include"]]
    cmd += ["-I" + i for i in incs] + ["-L" + l for l in libs]
    cmd += ["-L" + HERE, "-lwctb200", "-lc10", "-lc10_cuda", "-ltorch", "-ltorch_cpu", "-ltorch_cuda",
            "-ltorch_python", "-Wl,-rpath,$ORIGIN"] + ["-Wl,-rpath," + l for l in libs]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True, cwd=CSRC)
    os.replace(out + ".tmp", out)
    return out


if __name__ == "__main__":
    build(force=True, verbose=True)
    build_autograd(force=True, verbose=True)
