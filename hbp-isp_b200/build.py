"""Build the engine's shared library in-tree: hbp-isp_b200/lib/libhbp_b200.so.

    python hbp-isp_b200/build.py [--force]

Every CUDA source is compiled for sm_100a only. All kernels except the colour
conversion are compiled with --fmad=false: a*b+c is never contracted behind
the source's back, so the float arithmetic is exactly what the code spells out
(explicit __fmaf_rn where the reference's own build fuses), and the CPU oracle
(-ffp-contract=off) reproduces it bit for bit.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "lib")
OBJ = os.path.join(OUT, "obj")
LIB = os.path.join(OUT, "libhbp_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
BASE = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", f"-I{CSRC}", f"-I{os.path.join(ROOT, 'include')}"]
# files whose float arithmetic must not be contracted (everything but LAB)
CONTRACT_OK = {"lab.cu"}


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))


def headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(ROOT, "include", "hbp_b200.h"))
    return hs


def nvcc() -> str:
    for c in ("/usr/local/cuda/bin/nvcc", "nvcc"):
        if os.path.sep not in c or os.path.exists(c):
            return c
    return "nvcc"


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    hdr_time = max(os.path.getmtime(h) for h in headers())
    objs = []
    for s in sources():
        src = os.path.join(CSRC, s)
        obj = os.path.join(OBJ, s.replace(".cu", ".o"))
        objs.append(obj)
        if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr_time):
            continue
        flags = [] if s in CONTRACT_OK else ["--fmad=false"]
        cmd = [nvcc(), *ARCH, *BASE, *flags, "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose))
    sys.exit(0)
