"""TEST INFRASTRUCTURE ONLY: QUICK's own CUDA get2e, driven through its C ABI.

``oracle/_ref/refgpu_get2e`` is built from the reference's GPU sources where they
lie (``oracle/Makefile.refgpu``; s/p/d shells, the reference's own flags).  This
module writes one molecule, density and screen into the harness's input file,
runs the harness in its own process (QUICK's ``gpu_delete_`` resets the device)
and returns the reference's G and its timings.  Only tests and ``bench.py`` may
import it; nothing on the product path does.

The reference GPU path differs from the CPU get2e in two screens of its own: it
keeps only shell pairs with Y > 1e-10 (``src/gpu/cuda/gpu.cu:929-1030``) and
drops primitive-contracted integrals with |Y| below integralCutoff
(``src/gpu/gpu_get2e_subs.h:389``).  Its G therefore differs from the CPU
get2e's (and this library's) by the contributions of those quartets.

Input file layout (little-endian, in order): 12 int32 (natom, nbasis, nshell,
nprim, jbasis, maxcontract, MAXPRIM rows, nelec, charge, 0, 0, 0), 2 float64
(integralCutoff, primLimit), then the arrays of ``gpu_upload_xyz_``,
``gpu_upload_atom_and_chg_``, ``gpu_upload_basis_`` (Fortran order), Y
(nshell^2), cutPrim (jbasis^2), D (nbasis^2) and the density screen
(nshell^2).
"""
from __future__ import annotations

import json
import os
import shutil
import subprocess
import tempfile

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
BINARY = os.path.join(_HERE, "_ref", "refgpu_get2e")
# rows of gccoeff/gcexpo in the s/p/d reference build (src/gpu/gpu_common.h:39-41)
REF_MAXPRIM = 14


def available() -> bool:
    return os.path.exists(BINARY)


def build(ref_tree: str) -> None:
    """Compile the reference GPU get2e and the harness from ``ref_tree``."""
    subprocess.run(["make", "-s", "-f", os.path.join(_HERE, "Makefile.refgpu"), f"REF={ref_tree}"], check=True)


def _fort(a, dtype):
    return np.asarray(a, dtype=dtype).ravel(order="F")


def write_input(path, basis, D, cutmat, Y, cutprim, integral_cutoff, prim_limit):
    b = basis
    if b.has_f:
        raise ValueError("the reference GPU build here has s/p/d shells only")
    if int(b.kprim.max()) > REF_MAXPRIM:
        raise ValueError("a shell has more primitives than the reference build's MAXPRIM")
    mol = b.mol
    hdr = np.array([mol.natom, b.nbasis, b.nshell, b.nprim, b.jbasis, b.maxcontract, REF_MAXPRIM,
                    mol.nelec, int(getattr(mol, "charge", 0)), 0, 0, 0], dtype=np.int32)
    parts = [
        hdr, np.array([integral_cutoff, prim_limit], dtype=np.float64),
        np.ascontiguousarray(mol.xyz, dtype=np.float64).reshape(-1),   # xyz(3, natom), Bohr
        _fort(mol.Z, np.float64), _fort(mol.Z, np.int32),
        _fort(b.ncontract, np.int32), _fort(b.itype, np.int32), _fort(b.aexp, np.float64),
        _fort(b.dcoeff, np.float64), _fort(b.ncenter, np.int32), _fort(b.kstart, np.int32),
        _fort(b.katom, np.int32), _fort(b.ktype, np.int32), _fort(b.kprim, np.int32),
        _fort(b.ksumtype, np.int32), _fort(b.qnumber, np.int32), _fort(b.qstart, np.int32),
        _fort(b.qfinal, np.int32), _fort(b.qsbasis, np.int32), _fort(b.qfbasis, np.int32),
        _fort(b.gccoeff[:REF_MAXPRIM], np.float64), _fort(b.cons, np.float64),
        _fort(b.gcexpo[:REF_MAXPRIM], np.float64), _fort(b.klmn, np.int32),
        _fort(Y, np.float64), _fort(cutprim, np.float64), _fort(D, np.float64), _fort(cutmat, np.float64),
    ]
    with open(path, "wb") as f:
        for p in parts:
            f.write(np.ascontiguousarray(p).tobytes())


def run(basis, D, cutmat, Y, cutprim, integral_cutoff, prim_limit, steps=5, warmup=2, timeout=900):
    """G (nbasis x nbasis, symmetric) from QUICK's own GPU get2e, and its timings
    (``kernel_ms_*``: the get2e kernels alone, CUDA events; ``call_ms_*``: the
    whole per-build call sequence gpu_upload_calculated_ + gpu_upload_cutoff_ +
    gpu_get_cshell_eri_, host clock)."""
    if not available():
        raise FileNotFoundError(f"{BINARY} is not built (make -f oracle/Makefile.refgpu REF=...)")
    tmp = tempfile.mkdtemp(prefix="refgpu_")
    try:
        inp, out = os.path.join(tmp, "in.bin"), os.path.join(tmp, "G.bin")
        write_input(inp, basis, D, cutmat, Y, cutprim, integral_cutoff, prim_limit)
        r = subprocess.run([BINARY, inp, out, str(steps), str(warmup)], capture_output=True, text=True,
                           timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"refgpu harness failed ({r.returncode}): {r.stderr[-2000:]}")
        line = [ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1]
        info = json.loads(line)
        n = basis.nbasis
        G = np.fromfile(out, dtype=np.float64, count=n * n).reshape(n, n)
        return G, info
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
