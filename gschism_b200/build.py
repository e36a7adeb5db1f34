"""Build of the gschism_b200 native library (nvcc for sm_100a, in-tree).

Produces gschism_b200/_build/libgschism_b200.so from gschism_b200/csrc.  Per-file flags:
the backtracking and transport kernels are compiled with -fmad=false (bit-exact walk predicates,
limiter branches rounded like the CPU restatement), and host
code runs with FMA contraction off so the mesh geometry equals the CPU restatement.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(BUILD, "libgschism_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
NO_FMA = {"k_btrack.cu", "k_transport.cu"}


def _stale(out, deps):
    return (not os.path.exists(out)) or any(os.path.getmtime(d) > os.path.getmtime(out) for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = glob.glob(os.path.join(SRC, "*.h")) + glob.glob(os.path.join(SRC, "*.cuh")) + \
        [os.path.join(HERE, "..", "include", "gschism_b200.h")]
    objs = []
    for src in sorted(glob.glob(os.path.join(SRC, "*.cu")) + glob.glob(os.path.join(SRC, "*.cpp"))):
        name = os.path.basename(src)
        obj = os.path.join(BUILD, name + ".o")
        objs.append(obj)
        if not force and not _stale(obj, [src] + headers):
            continue
        if name.endswith(".cu"):
            cmd = [NVCC, "-c", src, "-o", obj, "-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
                   "-Xcompiler", "-ffp-contract=off", "--expt-relaxed-constexpr"] + ARCH
            if name in NO_FMA:
                cmd.append("-fmad=false")
        else:
            cmd = ["g++", "-c", src, "-o", obj, "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off",
                   "-I/usr/local/cuda/include"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        tmp = LIB + f".tmp{os.getpid()}"
        subprocess.run([NVCC, "-shared", "-o", tmp] + objs + ARCH + ["-cudart=static"], check=True)
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
