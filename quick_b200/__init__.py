"""quick_b200 -- B200-native closed-shell two-electron Fock build for QUICK.

The compute path is libquick_b200.so (hand-written CUDA for sm_100a behind the
C ABI in include/quick_b200.h); this package builds molecules and basis arrays
in QUICK's layout and drives the library.
"""
from .basis import Molecule, QuickBasis, build_basis  # noqa: F401

__all__ = ["Molecule", "QuickBasis", "build_basis"]
