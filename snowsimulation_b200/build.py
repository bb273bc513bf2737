"""Build libsnowb200.so in-tree for sm_100a with nvcc.

Flags: -fmad=false keeps every multiply and add separately rounded, and fast math stays off
so division and sqrt are correctly rounded -- the arithmetic contract shared with the CPU
oracle (and with the reference when it is built with the same IEEE settings).
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc", "snow_b200.cu")
OUT = os.path.join(HERE, "libsnowb200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-Xcompiler", "-fPIC", "-shared",
]


def sources():
    d = os.path.join(HERE, "csrc")
    return [os.path.join(d, f) for f in os.listdir(d) if f.endswith((".cu", ".cuh"))] + [
        os.path.join(HERE, "..", "include", "snow_b200.h")]


def up_to_date():
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(s) <= t for s in sources())


def build(force=False, verbose=False, extra=()):
    if not force and up_to_date():
        return OUT
    cmd = [NVCC, *NVCC_FLAGS, *extra, "-o", OUT, SRC]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else [])
