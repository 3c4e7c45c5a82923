"""Builds tests/compat/compat_demo.cpp against include/latfield2_b200.hpp and
liblf2gpu.so (no GPU needed to build):

    python tests/compat/build_demo.py [--single] [--out PATH]
"""
import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def build(out, single=False):
    sys.path.insert(0, ROOT)
    from latfield2_b200 import build as B
    lib = B.build()
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include"),
           os.path.join(HERE, "compat_demo.cpp"), "-o", out, "-L", os.path.dirname(lib), "-llf2gpu",
           "-Wl,-rpath," + os.path.dirname(lib)]
    if single:
        cmd.insert(1, "-DSINGLE")
    subprocess.run(cmd, check=True)
    return out


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--single", action="store_true")
    ap.add_argument("--out", default=os.path.join(HERE, "compat_demo"))
    a = ap.parse_args()
    print(build(a.out, a.single))
