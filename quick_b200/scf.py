"""Closed-shell SCF driver around the B200 Fock build.

The caller of the hot path, restated on the GPU: QUICK's ``electdiis`` +
``scf_operator`` (``src/modules/quick_scf_module.f90:165-802``,
``src/modules/quick_scf_operator_module.f90:26-250``):

* H = T + V from the device one-electron integrals (``qk_oei_host``);
* symmetric orthogonalisation X = S^-1/2 (``fullx``);
* each iteration F = H + G(D) through ``Get2e.fock2e``; from cycle ``ncyc``
  on (QUICK default 3, ``quick_method_module.f90:117``) the incremental form
  F = F_prev + G(D - D_prev) with the density screen taken on the difference
  (``quick_scf_operator_module.f90:69-82``);
* Pulay DIIS on FDS - SDF with up to 10 vectors;
* convergence when the RMS density change is below ``denserms`` and its largest
  element below 100 * ``denserms`` (QUICK's PRMS / PCHANGE test), after at
  least 3 cycles;
* energy Eel = tr(D (H + F)) / 2, Etot = Eel + nuclear repulsion.

Dense linear algebra runs in torch (cuSOLVER) on the same device and stream.
"""
from __future__ import annotations

import ctypes
import math
import time

import numpy as np

from . import _native
from ._native import check, lib
from .get2e import Get2e


def oei(basis, ext_charges=None, device=0):
    """S, T, V (nbasis^2 numpy) computed on the GPU."""
    b = basis
    n = b.nbasis
    S = np.zeros((n, n))
    T = np.zeros((n, n))
    V = np.zeros((n, n))
    Z = np.ascontiguousarray(b.mol.Z, dtype=np.float64)
    xyz = np.ascontiguousarray(b.xyz, dtype=np.float64)
    if ext_charges is not None:
        exyz = np.ascontiguousarray(np.asarray(ext_charges[0], dtype=np.float64).reshape(-1, 3))
        eq = np.ascontiguousarray(ext_charges[1], dtype=np.float64)
        nx = len(eq)
    else:
        exyz = np.zeros((1, 3))
        eq = np.zeros(1)
        nx = 0
    arrs = [np.asfortranarray(b.ncontract, dtype=np.int32), np.asfortranarray(b.itype, dtype=np.int32),
            np.asfortranarray(b.aexp, dtype=np.float64), np.asfortranarray(b.dcoeff, dtype=np.float64),
            np.asfortranarray(b.ncenter, dtype=np.int32)]
    P = lambda a: ctypes.c_void_p(a.ctypes.data)  # noqa: E731
    check(lib().qk_oei_host(int(device), b.mol.natom, P(xyz), P(Z), n, b.maxcontract, *[P(a) for a in arrs],
                            nx, P(exyz), P(eq), P(S), P(T), P(V)), "qk_oei_host")
    return S, T, V


def external_repulsion(mol, ext_charges):
    if ext_charges is None:
        return 0.0
    pos = np.asarray(ext_charges[0], dtype=np.float64).reshape(-1, 3)
    q = np.asarray(ext_charges[1], dtype=np.float64)
    e = 0.0
    for a in range(mol.natom):
        r = np.linalg.norm(pos - mol.xyz[a], axis=1)
        e += float(mol.Z[a]) * float((q / r).sum())
    return e


class RHF:
    """Restricted Hartree-Fock on one GPU with the B200 get2e."""

    def __init__(self, basis, device: int = 0, integral_cutoff: float = 1e-10, prim_limit: float = None,
                 ext_charges=None, engine: Get2e = None):
        import torch
        self.torch = torch
        self.basis = basis
        self.device = torch.device("cuda", device)
        prim_limit = 0.1 * integral_cutoff if prim_limit is None else prim_limit
        self.eng = engine if engine is not None else Get2e(basis, device=device, integral_cutoff=integral_cutoff,
                                                          prim_limit=prim_limit)
        S, T, V = oei(basis, ext_charges, device)
        dt = torch.float64
        self.S = torch.tensor(S, dtype=dt, device=self.device)
        self.H = torch.tensor(T + V, dtype=dt, device=self.device)
        w, U = torch.linalg.eigh(self.S)
        keep = w > 1e-8
        self.X = U[:, keep] / torch.sqrt(w[keep])
        self.nocc = basis.mol.nelec // 2
        self.Ecore = basis.mol.nuclear_repulsion() + external_repulsion(basis.mol, ext_charges)
        self.fock_builds = 0

    def density(self, F):
        e, C = self.torch.linalg.eigh(self.X.T @ F @ self.X)
        C = self.X @ C[:, : self.nocc]
        return 2.0 * C @ C.T

    def guess(self, kind="gwh"):
        if kind == "core":
            return self.density(self.H)
        d = self.torch.diagonal(self.H)
        F0 = 0.875 * self.S * (d[:, None] + d[None, :])
        F0.fill_diagonal_(0.0)
        F0 += self.torch.diag(d)
        return self.density(F0)

    def run(self, denserms: float = 1e-6, maxiter: int = 100, guess="gwh", incremental: bool = True,
            ncyc: int = 3, maxdiis: int = 10, D0=None, verbose=False):
        torch = self.torch
        D = D0.clone() if D0 is not None else self.guess(guess)
        errs, focks = [], []
        F_prev = D_prev = None
        t0 = time.perf_counter()
        history = []
        converged = False
        for it in range(1, maxiter + 1):
            if incremental and F_prev is not None and it >= ncyc:
                F = F_prev.clone()
                self.eng.fock2e(D - D_prev, o=F)
            else:
                F = self.H.clone()
                self.eng.fock2e(D, o=F)
            self.fock_builds += 1
            F_prev, D_prev = F, D
            Eel = 0.5 * float(torch.sum(D * (self.H + F)))
            err = F @ D @ self.S - self.S @ D @ F
            errs.append(self.X.T @ err @ self.X)
            focks.append(F)
            if len(errs) > maxdiis:
                errs.pop(0)
                focks.pop(0)
            nd = len(errs)
            E = torch.stack(errs).reshape(nd, -1)
            Bm = -torch.ones((nd + 1, nd + 1), dtype=torch.float64, device=self.device)
            Bm[:nd, :nd] = E @ E.T
            Bm[nd, nd] = 0.0
            rhs = torch.zeros(nd + 1, dtype=torch.float64, device=self.device)
            rhs[nd] = -1.0
            try:
                c = torch.linalg.solve(Bm, rhs)[:nd]
                Fd = torch.einsum("k,kij->ij", c, torch.stack(focks))
            except RuntimeError:
                Fd = F
            Dn = self.density(Fd)
            dD = Dn - D
            prms = float(torch.sqrt(torch.mean(dD * dD)))
            pchange = float(torch.abs(dD).max())
            history.append((it, Eel + self.Ecore, prms))
            if verbose:
                print(it, Eel + self.Ecore, prms, pchange)
            if it >= 3 and prms < denserms and pchange < 100 * denserms:
                converged = True
                break
            D = Dn
        torch.cuda.synchronize(self.device)
        return {"E": Eel + self.Ecore, "Eel": Eel, "Ecore": self.Ecore, "D": D, "F": F, "niter": it,
                "converged": converged, "seconds": time.perf_counter() - t0, "history": history}
