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
    r = np.sqrt(((mol.xyz[:, None, :] - pos[None, :, :]) ** 2).sum(axis=2))
    return float((mol.Z.astype(np.float64)[:, None] * q[None, :] / r).sum())


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

    def state(self, denserms: float = 1e-6, maxiter: int = 100, guess="gwh", incremental: bool = True,
              ncyc: int = 3, maxdiis: int = 10, D0=None):
        """A solve that advances one Fock build at a time (:class:`SCFState`)."""
        return SCFState(self, denserms, maxiter, guess, incremental, ncyc, maxdiis, D0)

    def run(self, denserms: float = 1e-6, maxiter: int = 100, guess="gwh", incremental: bool = True,
            ncyc: int = 3, maxdiis: int = 10, D0=None, verbose=False):
        t0 = time.perf_counter()
        st = self.state(denserms, maxiter, guess, incremental, ncyc, maxdiis, D0)
        while not st.done:
            Db, F = st.fock_input()
            self.eng.fock2e(Db, o=F)
            st.step(st.step_device().tolist())
            if verbose:
                print(*st.history[-1])
        self.torch.cuda.synchronize(self.device)
        r = st.result()
        r["seconds"] = time.perf_counter() - t0
        return r


class SCFState:
    """One RHF solve driven one Fock build at a time, all matrices on the device.

    The loop of :meth:`RHF.run` split at the Fock build, so that a server can
    advance many solves together with one batched build (``Get2eBatch``) per
    step and one host synchronisation for all of them:

    1. :meth:`fock_input` -> (density to contract, matrix to accumulate into):
       D and H on full builds, D - D_prev and F_prev from cycle ``ncyc`` on
       (QUICK's incremental build, ``quick_scf_operator_module.f90:69-82``);
    2. the caller adds G(density) into that matrix;
    3. :meth:`step_device` -> a 3-vector (Eel, PRMS, PCHANGE) on the device:
       energy, Pulay DIIS over at most ``maxdiis`` vectors
       (``quick_scf_module.f90:165-802``; a singular DIIS system falls back to
       the plain Fock matrix on the device, without a host check), and the new
       density;
    4. :meth:`step` takes those three numbers on the host and applies QUICK's
       convergence test (PRMS < denserms and PCHANGE < 100 denserms, at least 3
       cycles).
    """

    def __init__(self, rhf, denserms, maxiter, guess, incremental, ncyc, maxdiis, D0):
        self.rhf = rhf
        self.torch = rhf.torch
        self.denserms, self.maxiter = denserms, maxiter
        self.incremental, self.ncyc, self.maxdiis = incremental, ncyc, maxdiis
        self.D = D0.clone() if D0 is not None else rhf.guess(guess)
        self.errs, self.focks = [], []
        self.F = self.F_prev = self.D_prev = self.Dn = None
        self.it = 0
        self.done = False
        self.converged = False
        self.Eel = None
        self.history = []

    def fock_input(self):
        self.it += 1
        if self.incremental and self.F_prev is not None and self.it >= self.ncyc:
            self.F = self.F_prev.clone()
            return self.D - self.D_prev, self.F
        self.F = self.rhf.H.clone()
        return self.D, self.F

    def step_device(self):
        torch = self.torch
        r = self.rhf
        F, D = self.F, self.D
        r.fock_builds += 1
        self.F_prev, self.D_prev = F, D
        Eel = 0.5 * torch.sum(D * (r.H + F))
        err = F @ D @ r.S - r.S @ D @ F
        self.errs.append(r.X.T @ err @ r.X)
        self.focks.append(F)
        if len(self.errs) > self.maxdiis:
            self.errs.pop(0)
            self.focks.pop(0)
        nd = len(self.errs)
        E = torch.stack(self.errs).reshape(nd, -1)
        Bm = -torch.ones((nd + 1, nd + 1), dtype=torch.float64, device=r.device)
        Bm[:nd, :nd] = E @ E.T
        Bm[nd, nd] = 0.0
        rhs = torch.zeros(nd + 1, dtype=torch.float64, device=r.device)
        rhs[nd] = -1.0
        sol, info = torch.linalg.solve_ex(Bm, rhs)
        Fd = torch.einsum("k,kij->ij", sol[:nd], torch.stack(self.focks))
        ok = (info == 0) & torch.isfinite(Fd).all()
        Fd = torch.where(ok, Fd, F)
        self.Dn = r.density(Fd)
        dD = self.Dn - D
        return torch.stack([Eel, torch.sqrt(torch.mean(dD * dD)), torch.abs(dD).max()])

    def step(self, vals):
        Eel, prms, pchange = (float(v) for v in vals)
        self.Eel = Eel
        self.history.append((self.it, Eel + self.rhf.Ecore, prms))
        if self.it >= 3 and prms < self.denserms and pchange < 100 * self.denserms:
            self.converged = True
            self.done = True
        elif self.it >= self.maxiter:
            self.done = True
            self.D = self.Dn
        else:
            self.D = self.Dn

    def result(self):
        r = self.rhf
        return {"E": self.Eel + r.Ecore, "Eel": self.Eel, "Ecore": r.Ecore, "D": self.D, "F": self.F,
                "niter": self.it, "converged": self.converged, "history": self.history}
