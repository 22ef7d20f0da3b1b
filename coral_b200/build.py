"""Builds coral_b200/libcoral_b200.so (CUDA sm_100a + host C++) with nvcc.

usage: python -m coral_b200.build [--verbose-ptxas]
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libcoral_b200.so")
SOURCES = ["kernels.cu", "capi.cu", "noalloc.cu", "host_setup.cpp"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def build(verbose_ptxas: bool = False, force: bool = False) -> str:
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    deps = srcs + [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".hpp", ".cuh"))]
    deps.append(os.path.join(os.path.dirname(HERE), "include", "coral_b200.h"))
    if not force and os.path.exists(LIB):
        t = os.path.getmtime(LIB)
        if all(os.path.getmtime(p) <= t for p in deps):
            return LIB
    cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC,-O3",
           "-o", LIB, *srcs, "-lcudart"]
    if verbose_ptxas:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(verbose_ptxas="--verbose-ptxas" in sys.argv, force=True))
