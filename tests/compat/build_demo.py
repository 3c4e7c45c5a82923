"""Builds a demo of tests/compat/ (compat_demo.cpp, the particle path;
poisson_demo.cpp, the FFT path; device_physics_demo.cu, user physics on the
GPU) against include/latfield2_b200.hpp and liblf2gpu.so (no GPU needed to
build):

    python tests/compat/build_demo.py [--single] [--source NAME.cpp] [--out PATH]
"""
import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def build(out, single=False, source="compat_demo.cpp"):
    """.cpp sources build with g++; .cu sources (user physics on the GPU)
    with nvcc for sm_100a."""
    sys.path.insert(0, ROOT)
    from latfield2_b200 import build as B
    lib = B.build()
    if source.endswith(".cu"):
        cmd = [B.nvcc(), *B.ARCH, "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
               os.path.join(HERE, source), "-o", out, "-L", os.path.dirname(lib), "-llf2gpu",
               "-Xlinker", "-rpath=" + os.path.dirname(lib)]
    else:
        cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include"),
               os.path.join(HERE, source), "-o", out, "-L", os.path.dirname(lib), "-llf2gpu",
               "-Wl,-rpath," + os.path.dirname(lib)]
    if single:
        cmd.insert(1, "-DSINGLE")
    subprocess.run(cmd, check=True)
    return out


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--single", action="store_true")
    ap.add_argument("--source", default="compat_demo.cpp")
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    out = a.out or os.path.join(HERE, os.path.splitext(a.source)[0])
    print(build(out, a.single, a.source))
