"""Build recipe for the sm_100a shared library (koral_b200/_lib/libkoral_b200.so).

nvcc compiles the kernels for sm_100a only.  Physics device code is built
with --fmad=false (no fused multiply-add contraction) and IEEE division and
square root, and host code with -ffp-contract=off, so that arithmetic rounds
exactly as KORAL's x86-64 build does.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libkoral_b200.so")
SOURCES = ["kgpu.cu", "kgpu_setup.cu", "kgpu_diag.cu", "kgpu_avg.cu", "kgpu_noalloc.cu", "kgpu_rad.cu", "kgpu_mlp.cu",
           "kgpu_u2p_warm.cu"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "--fmad=false", "-prec-div=true", "-prec-sqrt=true",
    "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math",
    "-diag-suppress", "550",
]


def nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def build(verbose=False, ptxas_info=False):
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    deps = srcs + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    deps.append(os.path.join(HERE, "..", "include", "koral_b200.h"))
    if os.path.exists(LIB) and not ptxas_info:
        t = os.path.getmtime(LIB)
        if all(os.path.getmtime(d) <= t for d in deps):
            return LIB
    cmd = [nvcc()] + NVCC_FLAGS + (["-Xptxas", "-v"] if ptxas_info else []) + ["-shared", "-o", LIB] + srcs
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed")
    if ptxas_info or verbose:
        sys.stderr.write(r.stderr)
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_info="--ptxas" in sys.argv)
