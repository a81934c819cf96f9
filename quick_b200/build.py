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

# Device flags of every unit.  --split-compile: the device optimiser runs over the
# kernels of a unit in parallel (the class kernels are independent).
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [*ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", f"-DQK_MAX_L={MAX_L}",
              # kernel templates instantiated in one unit and launched from another (fock_lane_sp.cu)
              "-static-global-template-stub=false"]
# cuBLAS for the SP2 GEMMs of the SCF driver (scf.cu); in a process that has loaded
# torch, its libcublas.so.12 serves this dependency
LINK_FLAGS = [*ARCH, "-shared", "-lcublas", "-Xlinker", "-rpath=/usr/local/cuda/lib64"]
BUILD_DIR = os.path.join(HERE, "_build")


def units():
    """(source, extra flags) of the library's translation units.  The s/p per-lane
    kernels are a unit of their own compiled without a split: a split compile is not
    deterministic (two compiles of the same unit give different device code), and
    nvcc's code for these kernels varies with it by up to 15% in speed
    (fock_lane_sp.cu).  The rest is compiled with the split over all cores (without
    it, get2e.cu takes 13.5 minutes); its classes vary by a few percent."""
    return [(os.path.join(CSRC, "get2e.cu"), ["-DQK_LANE_SP_TU_SEPARATE", "--split-compile=0"]),
            (os.path.join(CSRC, "fock_lane_sp.cu"), []),
            (os.path.join(CSRC, "oei.cu"), []),
            (os.path.join(CSRC, "scf.cu"), [])]


def sources():
    return [u for u, _ in units()]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(BUILD_DIR, exist_ok=True)
    gen_dir = os.path.join(CSRC, "generated")
    subprocess.run([sys.executable, os.path.join(CSRC, "gen_eri.py"), gen_dir, str(MAX_L)],
                   check=True, stdout=subprocess.DEVNULL)
    deps = sources() + [os.path.join(gen_dir, "eri_classes.cuh"), os.path.join(CSRC, "common.cuh"),
                        os.path.join(ROOT, "include", "quick_b200.h"), os.path.abspath(__file__)]
    if not (force or _stale(LIB, deps)):
        return LIB
    inc = ["-I", os.path.join(ROOT, "include"), "-I", CSRC]
    objs, procs = [], []
    for src, extra in units():
        obj = os.path.join(BUILD_DIR, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        cmd = ["nvcc", *NVCC_FLAGS, *extra, *inc, "-c", "-o", obj, src]
        if verbose:
            print(" ".join(cmd))
        procs.append((cmd, subprocess.Popen(cmd)))
    for cmd, p in procs:
        if p.wait() != 0:
            raise subprocess.CalledProcessError(p.returncode, cmd)
    cmd = ["nvcc", *LINK_FLAGS, "-o", LIB, *objs]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
