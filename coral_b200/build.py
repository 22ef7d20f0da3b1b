"""Builds coral_b200/libcoral_b200.so (CUDA sm_100a + host C++) with nvcc.

Each source is compiled to its own object under coral_b200/_build (in
parallel, and only when it or a header is newer than its object), then the
objects are linked into the shared library.

usage: python -m coral_b200.build [--verbose-ptxas]
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcoral_b200.so")
SOURCES = ["kernels.cu", "capi.cu", "noalloc.cu", "host_setup.cpp", "zsplit.cu", "ensemble.cu", "closure.cu",
           "timeseries.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3"]


def _headers():
    hs = [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".hpp", ".cuh", ".h"))]
    hs.append(os.path.join(os.path.dirname(HERE), "include", "coral_b200.h"))
    return hs


def build(verbose_ptxas: bool = False, force: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    srcs = [s for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]
    hdr_t = max(os.path.getmtime(h) for h in _headers())
    jobs = []
    objs = []
    for s in srcs:
        src = os.path.join(CSRC, s)
        obj = os.path.join(OBJ, os.path.splitext(s)[0] + ".o")
        objs.append(obj)
        stale = force or not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(src), hdr_t)
        if stale:
            cmd = [NVCC, *ARCH, *FLAGS, "-c", "-o", obj, src]
            if verbose_ptxas and s.endswith(".cu"):
                cmd.insert(1, "-Xptxas=-v")
            jobs.append(cmd)

    def run(cmd):
        return subprocess.run(cmd, capture_output=True, text=True)

    if jobs:
        with ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as ex:
            res = list(ex.map(run, jobs))
        failed = False
        for cmd, r in zip(jobs, res):
            if r.stdout or r.stderr:
                sys.stderr.write(r.stdout + r.stderr)
            if r.returncode != 0:
                sys.stderr.write("failed: %s\n" % " ".join(cmd))
                failed = True
        if failed:
            raise subprocess.CalledProcessError(1, "nvcc")
    if jobs or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        subprocess.run([NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"], check=True)
    return LIB


if __name__ == "__main__":
    print(build(verbose_ptxas="--verbose-ptxas" in sys.argv, force="--force" in sys.argv))
