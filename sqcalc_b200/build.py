"""Build libsqnufft.so in-tree for sm_100a.

    python -m sqcalc_b200.build          # -> sqcalc_b200/libsqnufft.so
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libsqnufft.so")
SOURCES = ["sqn_api.cu", "sqn_kernels.cu", "sqn_fft512.cu", "sqn_adjoint.cu", "sqn_type1.cu",
           "sqn_noalloc.cu", "sqn_dump.cpp"]
HEADERS = ["sqn_internal.h", "sqn_device.cuh", os.path.join("..", "..", "include", "sqnufft.h")]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    exe = os.path.join(cuda, "bin", "nvcc")
    return exe if os.path.exists(exe) else (shutil.which("nvcc") or "nvcc")


def cuda_lib_dir():
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    return os.path.join(cuda, "lib64")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, extra=()):
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    deps = srcs + [os.path.join(CSRC, h) for h in HEADERS] + [__file__]
    if not force and not _stale(LIB, deps):
        return LIB
    libdir = cuda_lib_dir()
    cmd = [nvcc(), "-O3", "-std=c++17", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC", "-shared",
           "--expt-relaxed-constexpr", "-ccbin", "/usr/bin/g++" if os.path.exists("/usr/bin/g++")
           else "g++", *extra, "-o", LIB, *srcs, "-L" + libdir, "-lcufft", "-lcudart",
           "-Xlinker", "-rpath=" + libdir]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True, cwd=CSRC)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True,
                extra=("-Xptxas", "-v") if "--ptxas" in sys.argv else ()))
