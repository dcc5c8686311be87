"""Builds libaltopir_gpu.so in this directory: the CUDA kernels for sm_100a plus the host-side C ABI.

Run as a script (``python build.py``) or through ``build()``.  nvcc cross-compiles without a GPU.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libaltopir_gpu.so")
SOURCES = ["csrc/alto_engine.cu", "csrc/host_setup.cpp"]
DEPS = SOURCES + ["csrc/kernels.cuh", "csrc/limb_gemm.cuh", "csrc/limb_gemm2.cuh", "csrc/sm100.cuh", "csrc/modq.cuh",
                  "csrc/serving.cuh", "csrc/hint.cuh", "csrc/offline.cuh", "../include/altopir_gpu.h"]


def nvcc_path():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def command(out=LIB, extra=()):
    return [
        nvcc_path(), "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
        # the g++ on PATH: the environment's CC/CXX may name a wrapper without OpenMP support
        "-ccbin", "g++", "-Xcompiler", "-fPIC,-fopenmp", "-shared", "-o", out,
        *[os.path.join(HERE, s) for s in SOURCES], "-lgomp", *extra,
    ]


def up_to_date(out=LIB):
    if not os.path.exists(out):
        return False
    t = os.path.getmtime(out)
    return all(os.path.getmtime(os.path.join(HERE, d)) <= t for d in DEPS)


def build(force=False, verbose=False):
    if not force and up_to_date():
        return LIB
    cmd = command()
    res = subprocess.run(cmd, cwd=HERE, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + res.stdout + res.stderr)
    if verbose:
        print(res.stdout + res.stderr)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
