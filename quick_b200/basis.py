"""Molecules and Gaussian basis sets in QUICK's own array layout.

This module builds, from an element list, Bohr coordinates and a basis-set name,
exactly the arrays QUICK's Fortran side hands to ``gpu_upload_basis_``
(``src/gpu/cuda/gpu.cu:1782``): shell tables ``kstart/katom/ktype/kprim/Ksumtype``,
the angular-momentum ranges ``Qstart/Qfinal/Qsbasis/Qfbasis``, per-function
``gccoeff/gcexpo/cons/KLMN``, and the per-function normalised contraction
``aexp/dcoeff/itype`` used for one-electron integrals.

Conventions followed (all from the reference):

* shell construction, Cartesian component order and ``cons`` factors:
  ``src/basis.f90:389-760`` (d: xx, xy, yy, xz, yz, zz with sqrt(3) on the
  mixed ones; f: xxx, xxy, xyy, yyy, xxz, xyz, yyz, xzz, yzz, zzz with sqrt(5)
  and sqrt(15));
* primitive normalisation ``xnorm`` and contraction renormalisation
  ``xnewnorm``: ``src/subs/xnorm.f90:22-98``; note the reference applies
  ``xnewnorm`` to S, P, SP and D shells but not to F shells
  (``src/basis.f90:683-755``), which is reproduced here;
* ``normalize_basis`` for ``dcoeff``: ``src/modules/quick_basis_module.f90:385-424``;
* Angstrom to Bohr with ``BOHRS_TO_A = 0.52917720859``
  (``src/modules/quick_constants_module.f90:77-79``).

All index-valued arrays hold 1-based values, as the Fortran caller would.
"""
from __future__ import annotations

import json
import math
import os
from dataclasses import dataclass, field

import numpy as np

BOHRS_TO_A = 0.52917720859
A_TO_BOHRS = 1.0 / BOHRS_TO_A
PI = 3.14159265358979323846264338327950288
PITO3HALF = PI ** 1.5
# MAXPRIM of the f-enabled reference build (src/modules/quick_size_module.f90:39-43)
MAXPRIM = 20

SYMBOLS = ["", "H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne", "Na", "Mg",
           "Al", "Si", "P", "S", "Cl", "Ar", "K", "Ca", "Sc", "Ti", "V", "Cr", "Mn",
           "Fe", "Co", "Ni", "Cu", "Zn", "Ga", "Ge", "As", "Se", "Br", "Kr", "Rb",
           "Sr", "Y", "Zr", "Nb", "Mo", "Tc", "Ru", "Rh", "Pd", "Ag", "Cd", "In",
           "Sn", "Sb", "Te", "I"]
Z_OF = {s.upper(): i for i, s in enumerate(SYMBOLS) if s}

# Cartesian exponents and cons factors per shell type, in QUICK order
_D_KLMN = [(2, 0, 0), (1, 1, 0), (0, 2, 0), (1, 0, 1), (0, 1, 1), (0, 0, 2)]
_D_CONS = [1.0, math.sqrt(3.0), 1.0, math.sqrt(3.0), math.sqrt(3.0), 1.0]
_F_KLMN = [(3, 0, 0), (2, 1, 0), (1, 2, 0), (0, 3, 0), (2, 0, 1), (1, 1, 1),
           (0, 2, 1), (1, 0, 2), (0, 1, 2), (0, 0, 3)]
_S5 = math.sqrt(5.0)
_F_CONS = [1.0, _S5, _S5, 1.0, _S5, _S5 * math.sqrt(3.0), _S5, _S5, _S5, 1.0]
_P_KLMN = [(1, 0, 0), (0, 1, 0), (0, 0, 1)]

_BASIS_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "basis_data")
_BASIS_ALIASES = {"6-31G(D)": "6-31G*", "6-31G(D,P)": "6-31G**"}


def xnorm(a: float, i: int, j: int, k: int) -> float:
    """Primitive Cartesian normalisation (src/subs/xnorm.f90:22-58)."""
    val = (2.0 * a) ** ((i + j + k) / 2.0 + 0.75)
    gamma = 1.0
    for n in (i, j, k):
        for L in range(1, n + 1):
            gamma *= (n - L) + 0.5
    return val * PI ** (-0.75) * gamma ** (-0.5)


def _gamma_prod(i, j, k):
    g = 1.0
    for n in (i, j, k):
        for L in range(1, n + 1):
            g *= (n - L) + 0.5
    return g


def xnewnorm(i: int, j: int, k: int, coef, expo) -> float:
    """Contraction renormalisation (src/subs/xnorm.f90:61-98)."""
    xponent = -1.5 - (i + j + k)
    s = 0.0
    for c1, a1 in zip(coef, expo):
        for c2, a2 in zip(coef, expo):
            s += c1 * c2 * (a1 + a2) ** xponent
    return (s * _gamma_prod(i, j, k) * PITO3HALF) ** (-0.5)


def load_basis_data(name: str) -> dict:
    key = name.upper()
    key = _BASIS_ALIASES.get(key, key)
    fname = key.replace("*", "s") + ".json"
    path = os.path.join(_BASIS_DIR, fname)
    if not os.path.exists(path):
        raise ValueError(f"basis set {name!r} is not packaged (looked for {fname})")
    with open(path) as f:
        return json.load(f)["elements"]


@dataclass
class Molecule:
    """Atoms with nuclear charges and Bohr coordinates (natom x 3)."""
    Z: np.ndarray
    xyz: np.ndarray
    charge: int = 0

    @staticmethod
    def from_angstrom(symbols, coords_ang, charge=0) -> "Molecule":
        Z = np.array([Z_OF[s.upper()] for s in symbols], dtype=np.int32)
        xyz = np.asarray(coords_ang, dtype=np.float64) * A_TO_BOHRS
        return Molecule(Z=Z, xyz=xyz, charge=charge)

    @property
    def natom(self):
        return len(self.Z)

    @property
    def nelec(self):
        return int(self.Z.sum()) - self.charge

    def nuclear_repulsion(self) -> float:
        """Ecore without external charges (src/getEnergy.f90:68-84)."""
        i, j = np.triu_indices(self.natom, 1)
        r = np.sqrt(((self.xyz[i] - self.xyz[j]) ** 2).sum(axis=1))
        return float((self.Z[i].astype(np.float64) * self.Z[j] / r).sum())


@dataclass
class QuickBasis:
    """QUICK basis arrays (Fortran semantics: 1-based index values)."""
    mol: Molecule
    name: str
    nshell: int = 0
    nbasis: int = 0
    nprim: int = 0
    jbasis: int = 0          # number of primitive slots (aex entries)
    maxcontract: int = 1
    kstart: np.ndarray = field(default=None)
    katom: np.ndarray = field(default=None)
    ktype: np.ndarray = field(default=None)
    kprim: np.ndarray = field(default=None)
    ksumtype: np.ndarray = field(default=None)   # nshell+1
    qnumber: np.ndarray = field(default=None)
    qstart: np.ndarray = field(default=None)
    qfinal: np.ndarray = field(default=None)
    qsbasis: np.ndarray = field(default=None)    # (nshell, 4)
    qfbasis: np.ndarray = field(default=None)    # (nshell, 4)
    gccoeff: np.ndarray = field(default=None)    # (MAXPRIM, nbasis)
    gcexpo: np.ndarray = field(default=None)     # (MAXPRIM, nbasis)
    cons: np.ndarray = field(default=None)       # (nbasis,)
    klmn: np.ndarray = field(default=None)       # (3, nbasis)
    aex: np.ndarray = field(default=None)        # (jbasis,)
    # one-electron representation (normalize_basis)
    ncenter: np.ndarray = field(default=None)    # (nbasis,) 1-based atom
    ncontract: np.ndarray = field(default=None)  # (nbasis,)
    itype: np.ndarray = field(default=None)      # (3, nbasis)
    aexp: np.ndarray = field(default=None)       # (maxcontract, nbasis)
    dcoeff: np.ndarray = field(default=None)     # (maxcontract, nbasis)
    has_f: bool = False

    @property
    def xyz(self):
        return self.mol.xyz

    def n_qshell(self) -> int:
        return int((self.qfinal - self.qstart + 1).sum())


_ELEMENT_TEMPLATES = {}


def build_basis(mol: Molecule, name: str) -> QuickBasis:
    """QUICK's basis arrays for ``mol`` (src/basis.f90:389-830), assembled from
    per-element templates: every array of a molecule is the concatenation of its
    atoms' blocks (an atom's shells, functions and primitives are contiguous and
    their normalisation involves only that atom), so each element's block is
    computed once by :func:`_build_basis_direct` and reused with offsets."""
    i32 = np.int32
    parts = []
    for z in mol.Z:
        key = (name, int(z))
        t = _ELEMENT_TEMPLATES.get(key)
        if t is None:
            t = _build_basis_direct(Molecule(Z=np.array([int(z)], dtype=np.int32), xyz=np.zeros((1, 3))), name)
            _ELEMENT_TEMPLATES[key] = t
        parts.append(t)
    b = QuickBasis(mol=mol, name=name)
    b.nshell = sum(t.nshell for t in parts)
    b.nbasis = sum(t.nbasis for t in parts)
    b.jbasis = sum(t.jbasis for t in parts)
    b.nprim = sum(t.nprim for t in parts)
    b.maxcontract = max(t.maxcontract for t in parts)
    b.has_f = any(t.has_f for t in parts)
    jb = np.cumsum([0] + [t.jbasis for t in parts])
    nb = np.cumsum([0] + [t.nbasis for t in parts])
    cat = np.concatenate
    b.kstart = cat([t.kstart + jb[a] for a, t in enumerate(parts)]).astype(i32)
    b.katom = cat([np.full(t.nshell, a + 1, dtype=i32) for a, t in enumerate(parts)])
    for f in ("ktype", "kprim", "qnumber", "qstart", "qfinal"):
        setattr(b, f, cat([getattr(t, f) for t in parts]).astype(i32))
    b.qsbasis = cat([t.qsbasis for t in parts]).astype(i32)
    b.qfbasis = cat([t.qfbasis for t in parts]).astype(i32)
    b.ksumtype = cat([t.ksumtype[:-1] + nb[a] for a, t in enumerate(parts)] +
                     [np.array([b.nbasis + 1])]).astype(i32)
    b.gccoeff = np.concatenate([t.gccoeff for t in parts], axis=1)
    b.gcexpo = np.concatenate([t.gcexpo for t in parts], axis=1)
    b.cons = cat([t.cons for t in parts])
    b.klmn = np.concatenate([t.klmn for t in parts], axis=1).astype(i32)
    b.aex = cat([t.aex for t in parts])
    b.ncenter = cat([np.full(t.nbasis, a + 1, dtype=i32) for a, t in enumerate(parts)])
    b.ncontract = cat([t.ncontract for t in parts]).astype(i32)
    b.itype = np.concatenate([t.itype for t in parts], axis=1).astype(i32)
    b.aexp = np.zeros((b.maxcontract, b.nbasis))
    b.dcoeff = np.zeros((b.maxcontract, b.nbasis))
    for a, t in enumerate(parts):
        b.aexp[:t.maxcontract, nb[a]:nb[a + 1]] = t.aexp
        b.dcoeff[:t.maxcontract, nb[a]:nb[a + 1]] = t.dcoeff
    return b


def _build_basis_direct(mol: Molecule, name: str) -> QuickBasis:
    """Assemble QUICK's basis arrays for ``mol`` shell by shell (src/basis.f90:389-830)."""
    data = load_basis_data(name)
    shells = []   # (atom_index0, kind, prims)
    for ia, z in enumerate(mol.Z):
        sym = SYMBOLS[int(z)]
        if sym not in data:
            raise ValueError(f"element {sym} missing from basis {name}")
        for kind, prims in data[sym]:
            if kind == "G":
                raise ValueError("g shells are not supported (reference ierr 37)")
            shells.append((ia, kind, prims))
    nfun = {"S": 1, "P": 3, "SP": 4, "D": 6, "F": 10}
    ktype_of = {"S": 1, "P": 3, "SP": 4, "D": 6, "F": 10}
    nshell = len(shells)
    nbasis = sum(nfun[k] for _, k, _ in shells)
    jbasis = sum(len(p) for _, _, p in shells)
    maxcontract = max(len(p) for _, _, p in shells)
    if maxcontract > MAXPRIM:
        raise ValueError("contraction longer than MAXPRIM")

    b = QuickBasis(mol=mol, name=name)
    b.nshell, b.nbasis, b.jbasis, b.maxcontract = nshell, nbasis, jbasis, maxcontract
    b.nprim = sum(len(p) * nfun[k] for _, k, p in shells)
    i32 = np.int32
    b.kstart = np.zeros(nshell, i32)
    b.katom = np.zeros(nshell, i32)
    b.ktype = np.zeros(nshell, i32)
    b.kprim = np.zeros(nshell, i32)
    b.ksumtype = np.zeros(nshell + 1, i32)
    b.qnumber = np.zeros(nshell, i32)
    b.qstart = np.zeros(nshell, i32)
    b.qfinal = np.zeros(nshell, i32)
    b.qsbasis = np.zeros((nshell, 4), i32)
    b.qfbasis = np.zeros((nshell, 4), i32)
    b.gccoeff = np.zeros((MAXPRIM, nbasis))
    b.gcexpo = np.zeros((MAXPRIM, nbasis))
    b.cons = np.zeros(nbasis)
    b.klmn = np.zeros((3, nbasis), i32)
    b.aex = np.zeros(jbasis)
    gcs = np.zeros(jbasis)
    gcp = np.zeros(jbasis)
    gcd = np.zeros(jbasis)
    gcf = np.zeros(jbasis)

    jb = 0    # 0-based primitive slot
    nf = 0    # 0-based basis function
    for js, (ia, kind, prims) in enumerate(shells):
        npr = len(prims)
        A = [p[0] for p in prims]
        B = [p[1] for p in prims]
        b.kprim[js] = npr
        b.ktype[js] = ktype_of[kind]
        b.katom[js] = ia + 1
        b.kstart[js] = jb + 1
        b.ksumtype[js] = nf + 1
        for k in range(npr):
            b.aex[jb + k] = A[k]
        if kind == "S":
            b.qnumber[js], b.qstart[js], b.qfinal[js] = 0, 0, 0
            b.qsbasis[js, 0], b.qfbasis[js, 0] = 0, 0
            for k in range(npr):
                gcs[jb + k] = B[k]
            c = [B[k] * xnorm(A[k], 0, 0, 0) for k in range(npr)]
            s = xnewnorm(0, 0, 0, c, A)
            b.cons[nf] = 1.0
            b.gccoeff[:npr, nf] = [s * x for x in c]
            b.gcexpo[:npr, nf] = A
            nf += 1
        elif kind == "P":
            b.qnumber[js], b.qstart[js], b.qfinal[js] = 6, 1, 1
            b.qsbasis[js, 1], b.qfbasis[js, 1] = 0, 2
            for k in range(npr):
                gcp[jb + k] = B[k]
            c = [B[k] * xnorm(A[k], 1, 0, 0) for k in range(npr)]
            s = xnewnorm(1, 0, 0, c, A)
            for m in range(3):
                b.cons[nf] = 1.0
                b.klmn[m, nf] = 1
                b.gccoeff[:npr, nf] = [s * x for x in c]
                b.gcexpo[:npr, nf] = A
                nf += 1
        elif kind == "SP":
            C = [p[2] for p in prims]
            b.qnumber[js], b.qstart[js], b.qfinal[js] = 1, 0, 1
            b.qsbasis[js, 0], b.qfbasis[js, 0] = 0, 0
            b.qsbasis[js, 1], b.qfbasis[js, 1] = 1, 3
            for k in range(npr):
                gcs[jb + k] = B[k]
                gcp[jb + k] = C[k]
            c = [B[k] * xnorm(A[k], 0, 0, 0) for k in range(npr)]
            s = xnewnorm(0, 0, 0, c, A)
            b.cons[nf] = 1.0
            b.gccoeff[:npr, nf] = [s * x for x in c]
            b.gcexpo[:npr, nf] = A
            nf += 1
            c = [C[k] * xnorm(A[k], 1, 0, 0) for k in range(npr)]
            s = xnewnorm(1, 0, 0, c, A)
            for m in range(3):
                b.cons[nf] = 1.0
                b.klmn[m, nf] = 1
                b.gccoeff[:npr, nf] = [s * x for x in c]
                b.gcexpo[:npr, nf] = A
                nf += 1
        elif kind == "D":
            b.qnumber[js], b.qstart[js], b.qfinal[js] = 2, 2, 2
            b.qsbasis[js, 2], b.qfbasis[js, 2] = 0, 5
            for k in range(npr):
                gcd[jb + k] = B[k]
            cols = []
            for m in range(6):
                l, mm, n = _D_KLMN[m]
                b.klmn[:, nf + m] = (l, mm, n)
                b.cons[nf + m] = _D_CONS[m]
                cols.append([B[k] * xnorm(A[k], l, mm, n) for k in range(npr)])
                b.gcexpo[:npr, nf + m] = A
            # xx, xy, yy scaled with xnewnorm(2,0,0, coeffs of yy);
            # xz, yz, zz scaled with xnewnorm(1,1,0, coeffs of zz)  (basis.f90:620-632)
            s1 = xnewnorm(2, 0, 0, cols[2], A)
            s2 = xnewnorm(1, 1, 0, cols[5], A)
            for m in range(6):
                s = s1 if m < 3 else s2
                b.gccoeff[:npr, nf + m] = [s * x for x in cols[m]]
            nf += 6
        elif kind == "F":
            b.has_f = True
            b.qnumber[js], b.qstart[js], b.qfinal[js] = 3, 3, 3
            b.qsbasis[js, 3], b.qfbasis[js, 3] = 0, 9
            for k in range(npr):
                gcf[jb + k] = B[k]
            for m in range(10):
                l, mm, n = _F_KLMN[m]
                b.klmn[:, nf + m] = (l, mm, n)
                b.cons[nf + m] = _F_CONS[m]
                b.gccoeff[:npr, nf + m] = [B[k] * xnorm(A[k], l, mm, n) for k in range(npr)]
                b.gcexpo[:npr, nf + m] = A
            nf += 10
        jb += npr
    b.ksumtype[nshell] = nf + 1
    assert nf == nbasis and jb == jbasis

    # one-electron (normalize_basis) representation: src/basis.f90:895-1010 and
    # src/modules/quick_basis_module.f90:385-424
    b.ncenter = np.zeros(nbasis, i32)
    b.ncontract = np.zeros(nbasis, i32)
    b.itype = np.zeros((3, nbasis), i32)
    b.aexp = np.zeros((maxcontract, nbasis))
    b.dcoeff = np.zeros((maxcontract, nbasis))
    l = 0
    for js in range(nshell):
        kt = int(b.ktype[js])
        k0 = int(b.kstart[js]) - 1
        npr = int(b.kprim[js])
        for j in range(kt):
            b.ncenter[l] = b.katom[js]
            b.ncontract[l] = npr
            if kt == 3:
                b.itype[j, l] = 1
            elif kt == 4 and j > 0:
                b.itype[j - 1, l] = 1
            elif kt == 6:
                b.itype[:, l] = _D_KLMN[j]
            elif kt == 10:
                b.itype[:, l] = _F_KLMN[j]
            for ll in range(npr):
                b.aexp[ll, l] = b.aex[k0 + ll]
                if kt == 1:
                    d = gcs[k0 + ll]
                elif kt == 3:
                    d = gcp[k0 + ll]
                elif kt == 4:
                    d = gcs[k0 + ll] if j == 0 else gcp[k0 + ll]
                elif kt == 6:
                    d = gcd[k0 + ll]
                else:
                    d = gcf[k0 + ll]
                b.dcoeff[ll, l] = d
            l += 1
    for ib in range(nbasis):
        t = b.itype[:, ib]
        n = int(b.ncontract[ib])
        for c in range(n):
            b.dcoeff[c, ib] *= xnorm(b.aexp[c, ib], int(t[0]), int(t[1]), int(t[2]))
        xponent = -1.5 - int(t.sum())
        s = 0.0
        for c1 in range(n):
            for c2 in range(n):
                s += b.dcoeff[c1, ib] * b.dcoeff[c2, ib] * (b.aexp[c1, ib] + b.aexp[c2, ib]) ** xponent
        s = (s * _gamma_prod(int(t[0]), int(t[1]), int(t[2])) * PITO3HALF) ** (-0.5)
        b.dcoeff[:n, ib] *= s
    return b
