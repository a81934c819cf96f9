"""CPU checks of the C ABI library: it loads without a GPU and exports every
symbol include/quick_b200.h declares (no compute calls)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "quick_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b((?:gpu|qk)_\w+)\s*\(", src)))


def test_header_and_binding_agree():
    from quick_b200 import _native
    assert sorted(_native.EXPORTED) == declared_symbols()


def test_library_exports_every_declared_symbol():
    from quick_b200 import _native
    if not os.path.exists(_native.LIB_PATH):
        pytest.skip("library not built (run __graft_entry__.build())")
    lib = ctypes.CDLL(_native.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_status_strings_without_gpu():
    from quick_b200 import _native
    if not os.path.exists(_native.LIB_PATH):
        pytest.skip("library not built")
    L = _native.lib()
    assert L.qk_status_string(0) == b"ok"
    assert b"layout" in L.qk_status_string(106)
    assert L.qk_max_l() >= 2


def test_basis_layout_matches_reference_convention():
    """The kernels assume QUICK's Cartesian order and cons factors; the host checks
    them on upload.  Verify the basis builder produces exactly that layout."""
    import math
    from quick_b200.basis import build_basis
    from quick_b200.molecules import water_cluster
    b = build_basis(water_cluster(1, 3.0), "CC-PVTZ")
    for s in range(b.nshell):
        for L in range(b.qstart[s], b.qfinal[s] + 1):
            f0 = b.ksumtype[s] - 1 + b.qsbasis[s, L]
            k = 0
            for nz in range(L + 1):
                for ny in range(L + 1 - nz):
                    e = (L - nz - ny, ny, nz)
                    assert tuple(b.klmn[:, f0 + k]) == e
                    nnz = sum(1 for x in e if x)
                    exp = 1.0 if (L <= 1 or nnz == 1) else (math.sqrt(3) if L == 2 else
                                                          (math.sqrt(5) if nnz == 2 else math.sqrt(15)))
                    assert abs(b.cons[f0 + k] - exp) < 1e-14
                    k += 1
