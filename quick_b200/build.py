"""Build the CUDA library in-tree (sm_100a): quick_b200/_lib/libquick_b200.so."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libquick_b200.so")
MAX_L = 3

# --split-compile=0: the device optimiser runs over the kernels in parallel on all
# host cores (the class kernels are independent; the build takes half the time)
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC", "-shared", f"-DQK_MAX_L={MAX_L}", "--split-compile=0",
              # cuBLAS for the SP2 GEMMs of the SCF driver (scf.cu); in a process that
              # has loaded torch, its libcublas.so.12 serves this dependency
              "-lcublas", "-Xlinker", "-rpath=/usr/local/cuda/lib64"]


def sources():
    return [os.path.join(CSRC, "get2e.cu"), os.path.join(CSRC, "oei.cu"), os.path.join(CSRC, "scf.cu")]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    gen_dir = os.path.join(CSRC, "generated")
    subprocess.run([sys.executable, os.path.join(CSRC, "gen_eri.py"), gen_dir, str(MAX_L)],
                   check=True, stdout=subprocess.DEVNULL)
    deps = sources() + [os.path.join(gen_dir, "eri_classes.cuh"), os.path.join(CSRC, "common.cuh"),
                        os.path.join(ROOT, "include", "quick_b200.h"), os.path.abspath(__file__)]
    if force or _stale(LIB, deps):
        cmd = ["nvcc", *NVCC_FLAGS, "-I", os.path.join(ROOT, "include"), "-I", CSRC,
               "-o", LIB, *sources()]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
