"""Builds liblf2gpu.so (the CUDA kernels and the C ABI) in-tree for sm_100a.

Usage: python -m latfield2_b200.build   (or python latfield2_b200/build.py)
The library is written next to this file; nvcc cross-compiles without a GPU.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "liblf2gpu.so")
SOURCES = ["lf2_abi.cu", "lf2_store.cu", "lf2_move.cu", "lf2_move_pipe.cu", "lf2_deposit.cu",
           "lf2_deposit_full.cu", "lf2_field.cu", "lf2_noalloc.cu", "lf2_pm.cu", "lf2_fft.cu",
           "lf2_exchange.cu"]
HEADERS = ["lf2_common.cuh", "lf2_deposit_common.cuh", "lf2_internal.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) is False or os.path.exists(cand)):
            return cand
    return "nvcc"


def inputs():
    files = [os.path.join(CSRC, s) for s in SOURCES + HEADERS]
    files.append(os.path.join(ROOT, "include", "lf2gpu.h"))
    return files


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in inputs())


def build(force=False, verbose=False):
    """Compiles every source into liblf2gpu.so unless it is up to date."""
    if not force and up_to_date():
        return LIB
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
           "-Xcompiler", "-fPIC", "-shared", "-I", os.path.join(ROOT, "include"), "-I", CSRC,
           "-o", LIB + ".tmp"] + [os.path.join(CSRC, s) for s in SOURCES] + ["-lcufft"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
