"""Closed-shell SCF driver around the B200 Fock build.

The caller of the hot path, restated on the GPU: QUICK's ``electdiis`` +
``scf_operator`` (``src/modules/quick_scf_module.f90:165-802``,
``src/modules/quick_scf_operator_module.f90:26-250``):

* the starting density is QUICK's default SAD guess (``quick_b200.guess``;
  "gwh" and "core" are available);
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
from ._native import check, lib, own_stream
from .get2e import Get2e

# QUICK's level-shift controls (quick_method_module.f90:96-98): allowed from cycle
# 3 when the largest DIIS error element exceeds 0.1 and the HOMO-LUMO gap is
# below 0.2, which is then opened to 0.2.
LSHIFT_CYCLE, LSHIFT_ERR, LSHIFT_GAP = 3, 0.1, 0.2

# The tightest integral cutoff QUICK's SCF schedule reaches (adjust_Cutoff below).
FINAL_CUTOFF = 1e-11


def adjust_cutoff(prms: float, cut: float, prim: float):
    """QUICK's integral cutoff during the SCF (``adjust_Cutoff``,
    ``src/modules/quick_method_module.f90:1107-1129``, called after every cycle
    with the RMS density change, ``quick_scf_module.f90:679-680``): once PRMS is
    at or below 1e-5, 1e-6, 1e-7 the cutoff tightens to 1e-9, 1e-10, 1e-11 --
    each step only from a cutoff looser than 10^-8.5, 10^-9.5, 10^-10.5 -- and
    primLimit follows it down.  The three tests run in turn, so one call may take
    several steps.  Returns (integral cutoff, primLimit)."""
    for p, above, new in ((1e-5, 10.0 ** -8.5, 1e-9), (1e-6, 10.0 ** -9.5, 1e-10), (1e-7, 10.0 ** -10.5, 1e-11)):
        if prms <= p and cut > above:
            cut = new
            prim = min(cut, prim)
    return cut, prim


class CutoffSchedule:
    """The cutoffs of one solve on its engine.  Disabled: the engine's cutoffs
    hold throughout.  Enabled: the solve starts at the engine's cutoffs and
    tightens them by :func:`adjust_cutoff` after every cycle; the work lists are
    built once, at the final cutoff, before the first build (the builds apply the
    cutoff in force themselves, so the lists only have to hold every quartet it
    admits), and :meth:`restore` puts the starting cutoffs back.  As in QUICK the
    incremental builds carry on across a change (no full rebuild)."""

    def __init__(self, eng, enabled: bool):
        self.eng, self.enabled = eng, bool(enabled)
        self.start = (eng.integral_cutoff, eng.prim_limit)
        self.cut, self.prim = self.start
        self.changes = []
        if self.enabled:
            final = min(self.cut, FINAL_CUTOFF)
            if final < self.cut:
                eng.set_cutoffs(final, self.prim)
                eng.prepare()
                eng.set_cutoffs(self.cut, self.prim)

    def update(self, it: int, prms: float) -> bool:
        """Apply the schedule after cycle ``it``; True when the cutoffs changed."""
        if not self.enabled:
            return False
        cut, prim = adjust_cutoff(prms, self.cut, self.prim)
        if (cut, prim) == (self.cut, self.prim):
            return False
        self.cut, self.prim = cut, prim
        self.eng.set_cutoffs(cut, prim)
        self.changes.append((it, cut, prim))
        return True

    def restore(self) -> bool:
        """Put the starting cutoffs back; True when they had changed."""
        if self.enabled and (self.cut, self.prim) != self.start:
            self.eng.set_cutoffs(*self.start)
            self.cut, self.prim = self.start
            return True
        return False


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
        """Initial density: "core" (H), "gwh" (generalised Wolfsberg-Helmholz) or
        "sad" (superposition of atomic densities, quick_b200.guess)."""
        if kind == "sad":
            from .guess import sad_density
            return self.torch.tensor(sad_density(self.basis, self.device.index or 0), device=self.device)
        if kind == "core":
            return self.density(self.H)
        d = self.torch.diagonal(self.H)
        F0 = 0.875 * self.S * (d[:, None] + d[None, :])
        F0.fill_diagonal_(0.0)
        F0 += self.torch.diag(d)
        return self.density(F0)

    def state(self, denserms: float = 1e-6, maxiter: int = 100, guess="sad", incremental: bool = True,
              ncyc: int = 3, maxdiis: int = 10, D0=None, adaptive_cutoff: bool = False):
        """A solve that advances one Fock build at a time (:class:`SCFState`).
        ``adaptive_cutoff``: QUICK's cutoff schedule (:class:`CutoffSchedule`)."""
        return SCFState(self, denserms, maxiter, guess, incremental, ncyc, maxdiis, D0, adaptive_cutoff)

    def run(self, denserms: float = 1e-6, maxiter: int = 100, guess="sad", incremental: bool = True,
            ncyc: int = 3, maxdiis: int = 10, D0=None, verbose=False, adaptive_cutoff: bool = False):
        t0 = time.perf_counter()
        st = self.state(denserms, maxiter, guess, incremental, ncyc, maxdiis, D0, adaptive_cutoff)
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

    def __init__(self, rhf, denserms, maxiter, guess, incremental, ncyc, maxdiis, D0, adaptive_cutoff=False):
        self.rhf = rhf
        self.cutoffs = CutoffSchedule(rhf.eng, adaptive_cutoff)
        self.torch = rhf.torch
        self.denserms, self.maxiter = denserms, maxiter
        self.incremental, self.ncyc, self.maxdiis = incremental, ncyc, maxdiis
        self.warm = D0 is not None
        self.D = D0.clone() if D0 is not None else rhf.guess(guess)
        self.errs, self.focks = [], []
        self.F = self.F_prev = self.D_prev = self.Dn = None
        self.vec, self.gap = None, None    # previous eigenvectors (orthogonal basis), HOMO-LUMO gap
        self.shifts = 0
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
        # new density: diagonalise X^T Fd X, level-shifted as QUICK does
        # (quick_scf_module.f90:620-680): in the basis of the previous eigenvectors
        # the virtual levels move up by (0.2 - gap)
        Fo = r.X.T @ Fd @ r.X
        shift = 0.0
        if self.it >= LSHIFT_CYCLE and self.vec is not None and self.gap < LSHIFT_GAP:
            if float(torch.abs(err).max()) > LSHIFT_ERR:
                shift = LSHIFT_GAP - self.gap
        if shift > 0.0:
            Fo = self.vec.T @ Fo @ self.vec
            v = torch.arange(r.nocc, Fo.shape[0], device=r.device)
            Fo[v, v] += shift
            self.shifts += 1
        e, V = torch.linalg.eigh(Fo)
        if shift > 0.0:
            V = self.vec @ V
        self.vec = V
        ev = e[r.nocc - 1: r.nocc + 1].cpu() if r.nocc < e.shape[0] else None
        self.gap = float(ev[1] - ev[0]) if ev is not None else 1.0
        Co = r.X @ V[:, : r.nocc]
        self.Dn = 2.0 * Co @ Co.T
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
            self.cutoffs.update(self.it, prms)

    def result(self):
        r = self.rhf
        self.cutoffs.restore()
        return {"E": self.Eel + r.Ecore, "Eel": self.Eel, "Ecore": r.Ecore, "D": self.D, "F": self.F,
                "niter": self.it, "converged": self.converged, "history": self.history,
                "cutoff_changes": list(self.cutoffs.changes)}


def gershgorin_range(Fo) -> float:
    """Width of the Gershgorin interval of a symmetric matrix (the interval the
    SP2 projection maps onto [0, 1])."""
    import torch
    d = torch.diagonal(Fo)
    rad = torch.abs(Fo).sum(dim=1) - torch.abs(d)
    return float(torch.max(d + rad) - torch.min(d - rad))


def sp2_steps(eigvals, nocc: int, width: float = None) -> int:
    """SP2 projection steps for a spectrum ``eigvals`` (ascending) with ``nocc``
    occupied levels mapped from an interval of ``width`` (default: the spectral
    range): twice log2(2 width / HOMO-LUMO gap) -- the steps that open the gap --
    plus 28 for the quadratic end game (which takes 15-22 steps to reach 1e-12 on
    spectra of 60-600 levels), clamped to [30, 160]."""
    e = [float(x) for x in eigvals]
    gap = max(e[nocc] - e[nocc - 1], 1e-6) if 0 < nocc < len(e) else 1.0
    w = max(width if width is not None else e[-1] - e[0], 2.0 * gap)
    return int(min(160, max(30, math.ceil(2.0 * math.log2(2.0 * w / gap)) + 28)))


class GraphSCF:
    """RHF whose whole iteration -- Fock build, energy, Pulay DIIS and the new
    density -- is one CUDA graph, replayed once per cycle.

    What keeps the iteration free of host synchronisation:

    * the Fock build accumulates ``base + G(D - Dref)`` into a static matrix:
      ``base = H, Dref = 0`` for the full builds of the first cycles, and
      ``base = F_prev, Dref = D_prev`` afterwards (QUICK's incremental build,
      ``quick_scf_operator_module.f90:69-82``);
    * the DIIS history is a fixed set of ``maxdiis`` slots shifted each cycle,
      with the unused slots masked out of the B matrix by a device-side count,
      and the DIIS system is solved by ``qk_small_solve`` (partial pivoting in
      one warp; a vanishing pivot keeps the plain Fock matrix, as in
      :class:`SCFState`);
    * the density is the projector onto the ``nocc`` lowest levels of X^T F X by
      SP2 purification (Niklasson, Phys. Rev. B 66, 155115 (2002)): Y0 maps the
      Gershgorin interval onto [1, 0], then Y <- Y^2 or 2Y - Y^2, whichever trace
      is nearer nocc, a fixed number of steps (:func:`sp2_steps`, from the
      spectrum of the guess).  The projector is the same one diagonalisation
      gives; D = 2 X Y X^T.

    Each replay also writes (Eel, PRMS, PCHANGE) of the cycle; the host reads
    those three numbers for QUICK's convergence test.  ``graph=False`` runs the
    same body eagerly (same kernels, same numbers).
    """

    def __init__(self, rhf, maxdiis: int = 10, sp2: int = None):
        torch = rhf.torch
        self.rhf, self.torch = rhf, torch
        n, m, k = rhf.basis.nbasis, rhf.X.shape[1], maxdiis
        dev, dt = rhf.device, torch.float64
        z = lambda *s: torch.zeros(s, dtype=dt, device=dev)  # noqa: E731
        self.k, self.m = k, m
        self.D, self.Dref, self.base, self.F = z(n, n), z(n, n), z(n, n), z(n, n)
        self.errs, self.focks = z(k, m, m), z(k, n, n)
        self.valid = torch.zeros((), dtype=torch.int64, device=dev)
        self.idx = torch.arange(k, device=dev)
        self.B, self.rhs, self.c = z(k + 1, k + 1), z(k + 1), z(k + 1)
        self.rhs[k] = -1.0
        self.ok = torch.zeros(1, dtype=torch.int32, device=dev)
        self.eye_k = torch.eye(k, dtype=dt, device=dev)
        self.eye_m = torch.eye(m, dtype=dt, device=dev)
        self.Ya, self.Yb, self.Y2 = z(m, m), z(m, m), z(m, m)   # SP2 iterates (ping-pong) and Y Y
        # zero steps: creates the library's cuBLAS handle for the device now, outside
        # any graph capture (creating it inside one would allocate)
        check(lib().qk_sp2_run(ctypes.c_void_p(self.Ya.data_ptr()), ctypes.c_void_p(self.Yb.data_ptr()),
                               ctypes.c_void_p(self.Y2.data_ptr()), m, 0.0, 0,
                               ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)), "qk_sp2_run")
        self.out = z(4)
        self.cycle = torch.zeros((), dtype=torch.int64, device=dev)
        self.XtS = rhf.X.T @ rhf.S          # orthogonal-basis projector of D: (XtS) D (XtS)^T / 2
        self.zero = torch.zeros((), dtype=dt, device=dev)
        self.minus_one = torch.full((), -1.0, dtype=dt, device=dev)
        self.lshift = torch.full((), LSHIFT_GAP, dtype=dt, device=dev)
        self.recaptures = 0
        self.sp2 = sp2
        self.graph = None
        self.post_graph = None      # the post-build half alone, for the full-build cycles

    def _density(self, Fd, shift=None):
        torch = self.torch
        X = self.rhf.X
        Fo = X.T @ Fd @ X
        if shift is not None:
            # level shift on the device: the virtual space of the current density
            # moves up by `shift` (0 when no shift is due)
            P = 0.5 * (self.XtS @ self.D @ self.XtS.T)
            Fo = Fo + shift * (self.eye_m - P)
        d = torch.diagonal(Fo)
        rad = torch.abs(Fo).sum(dim=1) - torch.abs(d)
        emin, emax = torch.min(d - rad), torch.max(d + rad)
        ne = float(self.rhf.nocc)
        torch.div(emax * self.eye_m - Fo, emax - emin, out=self.Ya)
        # all steps in one call (each: the symmetric square and one fused
        # trace-test-and-update launch); the result is in Ya after an even count
        stream = ctypes.c_void_p(torch.cuda.current_stream(self.rhf.device).cuda_stream)
        m = self.Ya.shape[0]
        check(lib().qk_sp2_run(ctypes.c_void_p(self.Ya.data_ptr()), ctypes.c_void_p(self.Yb.data_ptr()),
                               ctypes.c_void_p(self.Y2.data_ptr()), m, ne, self.sp2, stream), "qk_sp2_run")
        Y = self.Ya if self.sp2 % 2 == 0 else self.Yb
        # idempotency defect tr(Y - Y^2): zero once the projection has converged
        self.out[3].copy_(torch.trace(Y) - torch.sum(Y * Y))
        return 2.0 * (X @ Y @ X.T)

    def _post(self):
        """Everything of a cycle after the Fock build (F holds base + G)."""
        torch = self.torch
        r, k = self.rhf, self.k
        stream = torch.cuda.current_stream(r.device)
        F, D = self.F, self.D
        Eel = 0.5 * torch.sum(D * (r.H + F))
        err = F @ D @ r.S - r.S @ D @ F
        e = r.X.T @ err @ r.X
        self.cycle.add_(1)
        shift = torch.where((self.cycle >= LSHIFT_CYCLE) & (torch.abs(err).max() > LSHIFT_ERR),
                            self.lshift, self.zero)
        self.errs.copy_(torch.roll(self.errs, -1, 0))
        self.errs[k - 1].copy_(e)
        self.focks.copy_(torch.roll(self.focks, -1, 0))
        self.focks[k - 1].copy_(F)
        self.valid.copy_(torch.clamp(self.valid + 1, max=k))
        live = self.idx >= (k - self.valid)
        E = self.errs.reshape(k, -1)
        self.B[:k, :k].copy_(torch.where(live[:, None] & live[None, :], E @ E.T, self.eye_k))
        side = torch.where(live, self.minus_one, self.zero)
        self.B[:k, k].copy_(side)
        self.B[k, :k].copy_(side)
        self.B[k, k].zero_()
        check(lib().qk_small_solve(ctypes.c_void_p(self.B.data_ptr()), ctypes.c_void_p(self.rhs.data_ptr()), k + 1,
                                   ctypes.c_void_p(self.c.data_ptr()), ctypes.c_void_p(self.ok.data_ptr()),
                                   ctypes.c_void_p(stream.cuda_stream)), "qk_small_solve")
        Fd = torch.einsum("k,kij->ij", self.c[:k], self.focks)
        Fd = torch.where((self.ok[0] == 1) & torch.isfinite(Fd).all(), Fd, F)
        Dn = self._density(Fd, shift)
        dd = Dn - D
        self.out[0].copy_(Eel)
        self.out[1].copy_(torch.sqrt(torch.mean(dd * dd)))
        self.out[2].copy_(torch.abs(dd).max())
        self.Dref.copy_(D)
        self.base.copy_(F)
        self.D.copy_(Dn)

    def _pre(self, full: bool):
        """The start of a cycle: F <- base (H and Dref = 0 on full builds); returns
        the density the Fock build contracts, D - Dref."""
        if full:
            self.base.copy_(self.rhf.H)
            self.Dref.zero_()
        self.F.copy_(self.base)
        return self.D - self.Dref

    def _body(self):
        r = self.rhf
        stream = self.torch.cuda.current_stream(r.device)
        dD = self._pre(False)
        r.eng.fock2e(dD, o=self.F, stream=stream)
        self._post()

    def begin(self, guess: str = "sad", D0=None):
        """Guess density (or D0), SP2 step count from the guess spectrum, empty
        DIIS history."""
        torch = self.torch
        r = self.rhf
        if guess == "sad" and D0 is None:
            D0 = r.guess("sad")
        # the guess spectrum: the SP2 step count (set by the first solve on this
        # molecule, raised by the defect check) and, without D0, the density
        if self.sp2 is None or D0 is None:
            if guess == "core":
                Fg = r.H
            else:
                dg = torch.diagonal(r.H)
                Fg = 0.875 * r.S * (dg[:, None] + dg[None, :])
                Fg.fill_diagonal_(0.0)
                Fg += torch.diag(dg)
            Fo = r.X.T @ Fg @ r.X
            e, C = torch.linalg.eigh(Fo)
            if self.sp2 is None:
                self.sp2 = sp2_steps(e.cpu().numpy(), r.nocc, gershgorin_range(Fo))
            if D0 is None:
                Co = r.X @ C[:, : r.nocc]
                D0 = 2.0 * Co @ Co.T
        self.D.copy_(D0)
        self.valid.zero_()
        self.cycle.zero_()
        self.errs.zero_()
        self.focks.zero_()

    def run(self, denserms: float = 1e-6, maxiter: int = 100, guess: str = "sad", ncyc: int = 3, D0=None,
            graph: bool = True, adaptive_cutoff: bool = False):
        torch = self.torch
        r = self.rhf
        t0 = time.perf_counter()
        st = DeviceSCFState(r, denserms=denserms, maxiter=maxiter, guess=guess, ncyc=ncyc, D0=D0, g=self,
                            adaptive_cutoff=adaptive_cutoff)
        replayed = False
        while not st.done:
            if graph and st.it + 1 >= ncyc:
                st.it += 1
                if self.graph is None:
                    torch.cuda.synchronize(r.device)
                    self.graph = torch.cuda.CUDAGraph()
                    with torch.cuda.graph(self.graph):
                        self._body()
                self.graph.replay()
                replayed = True
            else:
                dD, F = st.fock_input()
                r.eng.fock2e(dD, o=F)
                if graph:
                    # the full-build cycles: the post-build half as its own graph
                    if self.post_graph is None:
                        torch.cuda.synchronize(r.device)
                        self.post_graph = torch.cuda.CUDAGraph()
                        with torch.cuda.graph(self.post_graph):
                            self._post()
                    self.post_graph.replay()
                else:
                    st.step_device()
            st.step(self.out.cpu().numpy())
        torch.cuda.synchronize(r.device)
        res = st.result()
        res.update({"seconds": time.perf_counter() - t0, "sp2_steps": self.sp2, "graph": replayed,
                    "recaptures": self.recaptures})
        return res


class DeviceSCFState:
    """One RHF solve on the device, one Fock build at a time, with the arithmetic
    of :class:`GraphSCF` (fixed-slot DIIS solved on the device, SP2 density): no
    host synchronisation inside a cycle, so a server can advance many solves with
    one batched build and ONE synchronisation per step.  The protocol of
    :class:`SCFState`: ``fock_input`` -> (density, matrix to add G into);
    ``step_device`` -> the cycle's (Eel, PRMS, PCHANGE, SP2 defect) on the device;
    ``step(values)``; ``result()``."""

    _pools = {}

    def __init__(self, rhf, denserms=1e-6, maxiter=100, guess="sad", ncyc=3, D0=None, maxdiis=10, g=None,
                 graph: bool = False, adaptive_cutoff: bool = False, lane: int = 0):
        self.rhf = rhf
        self.cutoffs = CutoffSchedule(rhf.eng, adaptive_cutoff)
        self.g = g if g is not None else GraphSCF(rhf, maxdiis=maxdiis)
        # graph=True: the post-build half of a cycle is captured once and replayed
        # (one launch per solve and step instead of some hundred)
        self.use_graph = graph
        self.post_graph = None
        self.lane = lane            # the stream and graph memory pool its post-build graph uses
        self.g.begin(guess, D0)
        self.denserms, self.maxiter, self.ncyc = denserms, maxiter, ncyc
        self.warm = D0 is not None
        self.it = 0
        self.done = False
        self.converged = False
        self.Eel = None
        self.history = []

    def fock_input(self):
        self.it += 1
        dD = self.g._pre(self.it < self.ncyc)
        return dD, self.g.F

    @classmethod
    def _lane(cls, torch, dev, lane):
        """Lane ``lane`` of device ``dev``: (graph memory pool, stream).  The
        post-build graphs of one lane share its pool and replay one after another on
        its stream, which makes the sharing safe; different lanes' graphs run
        concurrently.  The pool is owned by a small anchor graph that lives as long
        as the process (a pool dies with its last graph)."""
        key = (str(dev), lane)
        if key not in cls._pools:
            main = torch.cuda.current_stream(dev)
            # the stream is this process's own (not one of torch's pool streams,
            # which other threads can be handed too: their work would land in a
            # capture)
            pool = torch.cuda.graph_pool_handle()
            cs = own_stream(dev.index if dev.index is not None else torch.cuda.current_device())
            x = torch.zeros(1, device=dev)
            anchor = torch.cuda.CUDAGraph()
            cs.wait_stream(main)
            with torch.cuda.stream(cs):
                # this thread's cuBLAS handle and the stream's workspace are
                # created outside any capture
                w = torch.ones((2, 4, 4), dtype=torch.float64, device=dev)
                torch.einsum("k,kij->ij", w[:, 0, 0], w) @ w[0]
                torch.cuda.synchronize(dev)
                anchor.capture_begin(pool=pool, capture_error_mode="thread_local")
                y = x + 1.0
                anchor.capture_end()
            main.wait_stream(cs)
            cls._pools[key] = (pool, cs, anchor, x, y)
        return cls._pools[key][:2]

    def _replay(self):
        """Capture the post-build half on this solve's lane (first call, or after
        a recapture is due) and enqueue its replay there.  The caller orders the
        lane after the Fock build and the next reader after the lane."""
        torch = self.rhf.torch
        pool, cs = self._lane(torch, self.rhf.device, self.lane)
        with torch.cuda.stream(cs):
            if self.post_graph is None:
                gr = torch.cuda.CUDAGraph()
                # thread_local: set-up threads may allocate while this thread captures
                gr.capture_begin(pool=pool, capture_error_mode="thread_local")
                self.g._post()
                gr.capture_end()
                self.post_graph = gr
            self.post_graph.replay()
        return cs

    def step_device(self):
        if not self.use_graph:
            self.g._post()
            return self.g.out
        torch = self.rhf.torch
        main = torch.cuda.current_stream(self.rhf.device)
        _, cs = self._lane(torch, self.rhf.device, self.lane)
        cs.wait_stream(main)
        main.wait_stream(self._replay())
        return self.g.out

    @staticmethod
    def step_many(states, join=None):
        """``step_device`` of many solves after one (batched) Fock build: every
        lane waits once for the build, each solve's post-build graph replays on its
        lane (lanes run concurrently), then ``join`` (default: the current stream)
        waits once per lane.  Returns the solves' (Eel, PRMS, PCHANGE, defect)
        vectors, stacked on ``join``."""
        if not states:
            return None
        torch = states[0].rhf.torch
        dev = states[0].rhf.device
        main = torch.cuda.current_stream(dev)
        join = main if join is None else join
        ev = main.record_event()
        lanes = {}
        for st in states:
            if st.lane not in lanes:
                _, cs = st._lane(torch, dev, st.lane)
                cs.wait_event(ev)
                lanes[st.lane] = cs
        for st in states:
            if st.use_graph:
                st._replay()
            else:
                with torch.cuda.stream(lanes[st.lane]):
                    st.g._post()
        for cs in lanes.values():
            join.wait_stream(cs)
        with torch.cuda.stream(join):
            return torch.stack([st.g.out for st in states])

    def step(self, vals):
        g, r = self.g, self.rhf
        Eel, prms, pchange, defect = (float(x) for x in vals)
        self.Eel = Eel
        r.fock_builds += 1
        self.history.append((self.it, Eel + r.Ecore, prms))
        if abs(defect) > 1e-9 * max(1, r.nocc) and g.sp2 < 200:
            g.sp2 += 16                 # the projection needs more steps for this spectrum
            g.graph = None
            g.post_graph = None
            self.post_graph = None
            g.recaptures += 1
        if self.it >= 3 and prms < self.denserms and pchange < 100 * self.denserms:
            self.converged = self.done = True
        elif self.it >= self.maxiter:
            self.done = True
        elif self.cutoffs.update(self.it, prms):
            g.graph = None              # a captured build holds the cutoffs it was captured with
            g.recaptures += 1

    def result(self):
        g, r = self.g, self.rhf
        if self.cutoffs.restore():
            g.graph = None
        D = g.Dref.clone() if self.converged else g.D.clone()
        return {"E": self.Eel + r.Ecore, "Eel": self.Eel, "Ecore": r.Ecore, "D": D, "F": g.F.clone(),
                "niter": self.it, "converged": self.converged, "history": self.history,
                "cutoff_changes": list(self.cutoffs.changes)}
