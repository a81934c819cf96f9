"""The per-element template assembly of build_basis gives exactly the arrays of
the shell-by-shell builder (same numbers, shapes and dtypes)."""
import dataclasses

import numpy as np
import pytest

from quick_b200.basis import _build_basis_direct, build_basis
from quick_b200.molecules import alkane, water_cluster


@pytest.mark.parametrize("name", ["STO-3G", "3-21G", "6-31G*", "6-31G**", "CC-PVDZ", "CC-PVTZ", "DEF2-TZVP"])
def test_template_assembly_equals_direct(name):
    for mol in (water_cluster(4, 6.5, seed=3), alkane(3)):
        a, b = build_basis(mol, name), _build_basis_direct(mol, name)
        for f in dataclasses.fields(a):
            x, y = getattr(a, f.name), getattr(b, f.name)
            if isinstance(x, np.ndarray):
                assert x.dtype == y.dtype and x.shape == y.shape and np.array_equal(x, y), (name, f.name)
            elif f.name != "mol":
                assert x == y, (name, f.name)
