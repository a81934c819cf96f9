"""SAD initial guess: a superposition of atomic densities.

QUICK starts its SCF from the SAD guess by default (``quick_method%SAD``,
``src/modules/quick_method_module.f90:101``): for every atom type it runs an
atomic SCF and places the atomic densities on the diagonal blocks of the
molecular density (``get_sad_density_matrix``,
``src/modules/quick_sad_guess_module.f90:240-270``).  The reference's atomic SCF
is unrestricted (``sad_uscf``, same file :290-868).  Here the atom is solved
spin-restricted with fractional occupations -- 2 electrons per level in aufbau
order, the last electrons spread evenly over the lowest partly filled set of
degenerate levels -- which keeps the atomic density spherical and needs only
the closed-shell build G(D) = J(D) - K(D)/2 this library provides.  The guess
only sets the starting point: converged energies do not depend on it.

Atomic densities are computed once per (element, basis, device) with the GPU
Fock build and one-electron integrals and cached.
"""
from __future__ import annotations

import numpy as np

from .basis import Molecule, build_basis

_ATOM_CACHE = {}


def _occupations(e, nel: float, tol: float = 1e-4):
    occ = np.zeros(len(e))
    left = float(nel)
    i = 0
    while left > 1e-12 and i < len(e):
        j = i
        while j + 1 < len(e) and abs(e[j + 1] - e[i]) < tol * max(1.0, abs(e[i])):
            j += 1
        g = j - i + 1
        take = min(left, 2.0 * g)
        occ[i:j + 1] = take / g
        left -= take
        i = j + 1
    return occ


def atom_density(Z: int, basis_name: str, device: int = 0, maxiter: int = 200, tol: float = 1e-9):
    """Spherically averaged, fractionally occupied RHF density of a neutral atom
    (nbasis x nbasis numpy array, the atom's basis functions in QUICK's order)."""
    key = (int(Z), basis_name, device)
    if key in _ATOM_CACHE:
        return _ATOM_CACHE[key]
    import torch
    from .get2e import Get2e
    from .scf import oei
    mol = Molecule(Z=np.array([int(Z)], dtype=np.int32), xyz=np.zeros((1, 3)))
    b = build_basis(mol, basis_name)
    S, T, V = oei(b, None, device)
    dev = torch.device("cuda", device)
    S_t = torch.tensor(S, device=dev)
    H = torch.tensor(T + V, device=dev)
    w, U = torch.linalg.eigh(S_t)
    keep = w > 1e-8
    X = U[:, keep] / torch.sqrt(w[keep])
    eng = Get2e(b, device=device, integral_cutoff=1e-12, prim_limit=1e-13)
    try:
        e, C = torch.linalg.eigh(X.T @ H @ X)
        occ = torch.tensor(_occupations(e.cpu().numpy(), Z), device=dev)
        Cm = X @ C
        D = (Cm * occ) @ Cm.T
        errs, focks = [], []
        for _ in range(maxiter):
            F = H.clone()
            eng.fock2e(D, o=F)
            err = X.T @ (F @ D @ S_t - S_t @ D @ F) @ X
            errs.append(err)
            focks.append(F)
            if len(errs) > 8:
                errs.pop(0)
                focks.pop(0)
            nd = len(errs)
            Ev = torch.stack(errs).reshape(nd, -1)
            B = -torch.ones((nd + 1, nd + 1), dtype=torch.float64, device=dev)
            B[:nd, :nd] = Ev @ Ev.T
            B[nd, nd] = 0.0
            rhs = torch.zeros(nd + 1, dtype=torch.float64, device=dev)
            rhs[nd] = -1.0
            sol, info = torch.linalg.solve_ex(B, rhs)
            Fd = torch.einsum("k,kij->ij", sol[:nd], torch.stack(focks)) if int(info) == 0 else F
            e, C = torch.linalg.eigh(X.T @ Fd @ X)
            occ = torch.tensor(_occupations(e.cpu().numpy(), Z), device=dev)
            Cm = X @ C
            Dn = (Cm * occ) @ Cm.T
            delta = float(torch.sqrt(torch.mean((Dn - D) ** 2)))
            D = Dn
            if delta < tol:
                break
        out = D.cpu().numpy()
    finally:
        eng.close()
    _ATOM_CACHE[key] = out
    return out


def sad_density(basis, device: int = 0):
    """Molecular SAD density (numpy, nbasis x nbasis): atomic densities on the
    diagonal blocks, in the atom order of ``basis``."""
    n = basis.nbasis
    D = np.zeros((n, n))
    # basis functions of atom a: the shells with katom == a + 1, contiguous in QUICK's order
    f0 = np.asarray(basis.ksumtype[:-1], dtype=np.int64) - 1
    f1 = np.asarray(basis.ksumtype[1:], dtype=np.int64) - 1
    katom = np.asarray(basis.katom, dtype=np.int64) - 1
    for a in range(basis.mol.natom):
        sh = np.nonzero(katom == a)[0]
        if len(sh) == 0:
            continue
        lo, hi = int(f0[sh[0]]), int(f1[sh[-1]])
        Da = atom_density(int(basis.mol.Z[a]), basis.name, device)
        if Da.shape[0] != hi - lo:
            raise ValueError("atom basis block size mismatch")
        D[lo:hi, lo:hi] = Da
    return D
