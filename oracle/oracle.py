"""CPU ORACLE (test infrastructure only) -- ctypes front end and RHF driver.

Loads ``oracle/_build/liboracle.so`` (the C++ restatement of QUICK's CPU get2e,
see ``oracle.cpp``) and adds a numpy closed-shell SCF used to pin the oracle
against the reference's saved RHF energies (``test/saved/ene_*_rhf_*.out``).
Only tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU baseline and
reference arm may import this module.

SCF restated from ``src/modules/quick_scf_module.f90:165-802`` in its essentials:
symmetric orthogonalisation (``fullx``), Pulay DIIS on FDS-SDF, closed-shell
density D = 2 C_occ C_occ^T, electronic energy (tr(D H) + tr(D F)) / 2
(``eri.fh:1064-1083``) and total energy Eel + Ecore (``src/getEnergy.f90:152``).
The initial guess is the core Hamiltonian (or generalised Wolfsberg-Helmholz)
instead of SAD: the converged energy does not depend on it as long as the SCF
lands in the same state.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_V3 = os.path.join(_HERE, "_build", "liboracle.so")       # AVX2/FMA (x86-64-v3)
_LIB_V4 = os.path.join(_HERE, "_build", "liboracle_v4.so")    # AVX-512 (x86-64-v4)
_lib = None


def build():
    subprocess.run(["make", "-C", _HERE, "-s"], check=True)


def host_isa() -> str:
    """'v4' when the host CPU has the AVX-512 subsets of x86-64-v4, else 'v3'."""
    try:
        flags = set()
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("flags"):
                    flags = set(ln.split(":", 1)[1].split())
                    break
        return "v4" if {"avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl"} <= flags else "v3"
    except OSError:
        return "v3"


def lib_path() -> str:
    return _LIB_V4 if host_isa() == "v4" else _LIB_V3


def lib():
    global _lib
    if _lib is None:
        path = lib_path()
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        P = ctypes.c_void_p
        I = ctypes.c_int
        D = ctypes.c_double
        L.orc_create.restype = P
        L.orc_create.argtypes = [I, P, I, I, I] + [P] * 13
        L.orc_destroy.argtypes = [P]
        L.orc_boys.argtypes = [I, D, P]
        L.orc_set_boys_mode.argtypes = [I]
        L.orc_set_boys_mode.restype = I
        L.orc_schwarz.argtypes = [P, P, P, I]
        L.orc_density_cutoff.argtypes = [P, P, P]
        L.orc_get2e.restype = ctypes.c_longlong
        L.orc_get2e.argtypes = [P, P, P, P, P, D, D, P, I, I, I, I, I]
        L.orc_oei.argtypes = [I, I, P, P, P, P, P, P, I, P, P, P, P, P]
        L.orc_get2e_uhf.restype = ctypes.c_longlong
        L.orc_get2e_uhf.argtypes = [P, P, P, P, P, P, D, D, P, P, I]
        L.orc_density_cutoff_uhf.argtypes = [P, P, P, P]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _f64(a):
    return np.asfortranarray(a, dtype=np.float64)


def _i32(a):
    return np.asfortranarray(a, dtype=np.int32)


class quick_boys:
    """Context manager: the oracle's integrals use QUICK's own Boys function
    (a restatement of src/subs/fmt.f90, first order in X below X = 0.1) instead of
    the accurate one, to reproduce the reference's numbers to the last digits."""

    def __enter__(self):
        self.old = lib().orc_set_boys_mode(1)
        return self

    def __exit__(self, *exc):
        lib().orc_set_boys_mode(self.old)
        return False


def boys(M: int, T: float) -> np.ndarray:
    out = np.zeros(M + 2)
    lib().orc_boys(M, float(T), _p(out))
    return out[: M + 1]


class Oracle:
    """get2e oracle bound to one molecule + basis (QUICK array layout)."""

    def __init__(self, basis):
        self.b = basis
        b = basis
        self._keep = [np.ascontiguousarray(b.xyz, dtype=np.float64), _i32(b.kstart), _i32(b.katom),
                      _i32(b.ktype), _i32(b.kprim), _i32(b.ksumtype), _i32(b.qstart),
                      _i32(b.qfinal), _i32(b.qsbasis), _i32(b.qfbasis), _f64(b.gccoeff),
                      _f64(b.gcexpo), _f64(b.cons), _i32(b.klmn)]
        k = self._keep
        self.h = lib().orc_create(b.mol.natom, _p(k[0]), b.nshell, b.nbasis, b.jbasis,
                                  *[_p(x) for x in k[1:]])

    def __del__(self):
        try:
            if getattr(self, "h", None):
                lib().orc_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def schwarz(self, nthreads: int = 0):
        b = self.b
        Y = np.zeros((b.nshell, b.nshell), order="F")
        cp = np.zeros((b.jbasis, b.jbasis), order="F")
        lib().orc_schwarz(self.h, _p(Y), _p(cp), nthreads)
        return Y, cp

    def density_cutoff(self, D):
        b = self.b
        D = _f64(D)
        cm = np.zeros((b.nshell, b.nshell), order="F")
        lib().orc_density_cutoff(self.h, _p(D), _p(cm))
        return cm

    def get2e(self, D, cutmatrix, Ycut, cutprim, integral_cutoff, prim_limit, o=None,
              ii_range=(0, 0), nthreads=0, ii_stride=1, gpu_screens=False):
        """Return ``o + G(D)`` (symmetric, nbasis x nbasis) and the quartet count.

        ``gpu_screens``: also apply the two screens of QUICK's GPU path (shell pairs
        with Y <= 1e-10 left out, integrals with |Y| <= integral_cutoff not
        digested), to compare with that implementation."""
        b = self.b
        D = _f64(D)
        out = np.zeros((b.nbasis, b.nbasis), order="F") if o is None else _f64(o).copy(order="F")
        nq = lib().orc_get2e(self.h, _p(D), _p(_f64(cutmatrix)), _p(_f64(Ycut)), _p(_f64(cutprim)),
                             float(integral_cutoff), float(prim_limit), _p(out),
                             int(ii_range[0]), int(ii_range[1]), int(nthreads), int(ii_stride),
                             int(bool(gpu_screens)))
        return out, nq


def _uhf_methods():
    def density_cutoff_uhf(self, Da, Db):
        """QUICK's open-shell density screen (max of |Da + Db|, |Da|, |Db| per shell pair)."""
        b = self.b
        cm = np.zeros((b.nshell, b.nshell), order="F")
        lib().orc_density_cutoff_uhf(self.h, _p(_f64(Da)), _p(_f64(Db)), _p(cm))
        return cm

    def get2e_uhf(self, Da, Db, cutmatrix, Ycut, cutprim, integral_cutoff, prim_limit, nthreads=0):
        """(G_alpha, G_beta, quartet count) of the open-shell build (eri.fh under OSHELL)."""
        b = self.b
        oa = np.zeros((b.nbasis, b.nbasis), order="F")
        ob = np.zeros((b.nbasis, b.nbasis), order="F")
        nq = lib().orc_get2e_uhf(self.h, _p(_f64(Da)), _p(_f64(Db)), _p(_f64(cutmatrix)), _p(_f64(Ycut)),
                                 _p(_f64(cutprim)), float(integral_cutoff), float(prim_limit), _p(oa), _p(ob),
                                 int(nthreads))
        return oa, ob, nq

    Oracle.density_cutoff_uhf = density_cutoff_uhf
    Oracle.get2e_uhf = get2e_uhf


_uhf_methods()


def oei(basis, ext_charges=None):
    """Overlap, kinetic and nuclear-attraction matrices (with optional point charges)."""
    b = basis
    n = b.nbasis
    S = np.zeros((n, n), order="F")
    T = np.zeros((n, n), order="F")
    V = np.zeros((n, n), order="F")
    cx = [np.asarray(b.xyz, dtype=np.float64)]
    cq = [np.asarray(b.mol.Z, dtype=np.float64)]
    if ext_charges is not None:
        cx.append(np.asarray(ext_charges[0], dtype=np.float64).reshape(-1, 3))
        cq.append(np.asarray(ext_charges[1], dtype=np.float64))
    cxyz = np.ascontiguousarray(np.concatenate(cx))
    cchg = np.ascontiguousarray(np.concatenate(cq))
    keep = [_i32(b.ncontract), _i32(b.itype), _f64(b.aexp), _f64(b.dcoeff), _i32(b.ncenter),
            np.ascontiguousarray(b.xyz, dtype=np.float64)]
    lib().orc_oei(n, b.maxcontract, *[_p(x) for x in keep], len(cchg), _p(cxyz), _p(cchg),
                  _p(S), _p(T), _p(V))
    return S, T, V


def orthogonalizer(S, lindep=1e-8):
    w, U = np.linalg.eigh(S)
    keep = w > lindep
    return U[:, keep] / np.sqrt(w[keep])


def rhf(basis, integral_cutoff=1e-11, prim_limit=1e-12, conv=1e-9, maxiter=100, nthreads=0,
        ext_charges=None, fock_builder=None, verbose=False, guess="core"):
    """Closed-shell SCF; returns dict(E, Eel, Ecore, D, F, niter).

    ``fock_builder(D, cutmatrix) -> G`` may replace the oracle's get2e (used to
    run the same SCF with the CUDA Fock build)."""
    b = basis
    S, T, V = oei(b, ext_charges)
    H = T + V
    X = orthogonalizer(S)
    nocc = b.mol.nelec // 2
    orc = Oracle(b)
    Ycut, cutprim = orc.schwarz(nthreads)

    def G_of(D):
        cm = orc.density_cutoff(D)
        if fock_builder is not None:
            return fock_builder(D, cm)
        G, _ = orc.get2e(D, cm, Ycut, cutprim, integral_cutoff, prim_limit, nthreads=nthreads)
        return G

    def density(F):
        e, C = np.linalg.eigh(X.T @ F @ X)
        C = X @ C
        return 2.0 * C[:, :nocc] @ C[:, :nocc].T

    if isinstance(guess, np.ndarray):
        D = guess
    elif guess == "gwh":
        # generalised Wolfsberg-Helmholz: F_ij = 0.875 S_ij (H_ii + H_jj)
        d = np.diag(H)
        F0 = 0.875 * S * (d[:, None] + d[None, :])
        np.fill_diagonal(F0, d)
        D = density(F0)
    else:
        D = density(H)
    Ecore = b.mol.nuclear_repulsion()
    if ext_charges is not None:
        pos = np.asarray(ext_charges[0]).reshape(-1, 3)
        q = np.asarray(ext_charges[1])
        for a in range(b.mol.natom):
            r = np.linalg.norm(pos - b.xyz[a], axis=1)
            Ecore += float(b.mol.Z[a]) * float((q / r).sum())
    errs, focks = [], []
    E_old = 0.0
    for it in range(1, maxiter + 1):
        F = H + G_of(D)
        Eel = 0.5 * float(np.sum(D * (H + F)))
        err = F @ D @ S - S @ D @ F
        errs.append(X.T @ err @ X)
        focks.append(F)
        if len(errs) > 10:
            errs.pop(0)
            focks.pop(0)
        nd = len(errs)
        Bm = -np.ones((nd + 1, nd + 1))
        Bm[nd, nd] = 0.0
        for i in range(nd):
            for j in range(nd):
                Bm[i, j] = float(np.sum(errs[i] * errs[j]))
        rhs = np.zeros(nd + 1)
        rhs[nd] = -1.0
        try:
            c = np.linalg.solve(Bm, rhs)[:nd]
            Fd = sum(ci * Fi for ci, Fi in zip(c, focks))
        except np.linalg.LinAlgError:
            Fd = F
        Dn = density(Fd)
        dmax = float(np.abs(Dn - D).max())
        if verbose:
            print(it, Eel + Ecore, dmax, float(np.abs(errs[-1]).max()))
        converged = dmax < conv and abs(Eel - E_old) < 1e-10
        D_prev = D
        D = Dn
        E_old = Eel
        if converged:
            D = D_prev
            break
    return dict(E=Eel + Ecore, Eel=Eel, Ecore=Ecore, D=D, F=F, H=H, S=S, niter=it)


def uhf(basis, mult, integral_cutoff=1e-11, prim_limit=1e-12, conv=1e-9, maxiter=200, nthreads=0,
        fock_builder=None, guess="core"):
    """Unrestricted (Pople-Nesbet) SCF with QUICK's open-shell Fock build; returns
    dict(E, Da, Db, niter).  ``fock_builder(Da, Db, cutmatrix) -> (Ga, Gb)`` may
    replace the oracle's get2e_uhf.  Energy: (tr[(Da + Db) H] + tr[Da Fa] + tr[Db Fb]) / 2
    plus the nuclear repulsion; Pulay DIIS on the stacked alpha and beta commutators
    (the reference's uscf, src/modules/quick_uscf_module.f90, in its essentials)."""
    b = basis
    S, T, V = oei(b)
    H = T + V
    X = orthogonalizer(S)
    nel = b.mol.nelec
    na, nb = (nel + mult - 1) // 2, (nel - mult + 1) // 2
    orc = Oracle(b)
    Ycut, cutprim = orc.schwarz(nthreads)

    def G_of(Da, Db):
        cm = orc.density_cutoff_uhf(Da, Db)
        if fock_builder is not None:
            return fock_builder(Da, Db, cm)
        Ga, Gb, _ = orc.get2e_uhf(Da, Db, cm, Ycut, cutprim, integral_cutoff, prim_limit, nthreads)
        return Ga, Gb

    def dens(F, nocc):
        e, C = np.linalg.eigh(X.T @ F @ X)
        C = X @ C
        return C[:, :nocc] @ C[:, :nocc].T

    Da, Db = dens(H, na), dens(H, nb)
    Ecore = b.mol.nuclear_repulsion()
    errs, focks = [], []
    E_old = 0.0
    for it in range(1, maxiter + 1):
        Ga, Gb = G_of(Da, Db)
        Fa, Fb = H + Ga, H + Gb
        Eel = 0.5 * float(np.sum((Da + Db) * H) + np.sum(Da * Fa) + np.sum(Db * Fb))
        ea = X.T @ (Fa @ Da @ S - S @ Da @ Fa) @ X
        eb = X.T @ (Fb @ Db @ S - S @ Db @ Fb) @ X
        errs.append((ea, eb))
        focks.append((Fa, Fb))
        if len(errs) > 10:
            errs.pop(0)
            focks.pop(0)
        nd = len(errs)
        Bm = -np.ones((nd + 1, nd + 1))
        Bm[nd, nd] = 0.0
        for i in range(nd):
            for j in range(nd):
                Bm[i, j] = float(np.sum(errs[i][0] * errs[j][0]) + np.sum(errs[i][1] * errs[j][1]))
        rhs = np.zeros(nd + 1)
        rhs[nd] = -1.0
        try:
            c = np.linalg.solve(Bm, rhs)[:nd]
            Fa_d = sum(ci * f[0] for ci, f in zip(c, focks))
            Fb_d = sum(ci * f[1] for ci, f in zip(c, focks))
        except np.linalg.LinAlgError:
            Fa_d, Fb_d = Fa, Fb
        Dan, Dbn = dens(Fa_d, na), dens(Fb_d, nb)
        dmax = max(float(np.abs(Dan - Da).max()), float(np.abs(Dbn - Db).max()))
        converged = dmax < conv and abs(Eel - E_old) < 1e-10
        Da_prev, Db_prev = Da, Db
        Da, Db = Dan, Dbn
        E_old = Eel
        if converged:
            Da, Db = Da_prev, Db_prev
            break
    return dict(E=Eel + Ecore, Eel=Eel, Ecore=Ecore, Da=Da, Db=Db, niter=it)
