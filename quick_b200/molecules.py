"""Seeded synthetic molecules for the get2e workloads.

* ``water_cluster(n, box)`` -- n rigid waters (O-H 0.96 A, H-O-H 104.5 deg),
  uniformly random orientations (uniform unit quaternions), oxygens uniform in
  a ``box`` Angstrom cube, rejecting placements with an O-O distance < 2.8 A.
* ``alkane(n)`` -- linear all-trans CnH(2n+2) with C-C 1.54 A, C-H 1.09 A,
  tetrahedral angles, and per-atom Gaussian jitter (sigma 0.02 A).

All generators use numpy's PCG64 with an explicit seed, so a workload is fully
named by (kind, size, seed).
"""
from __future__ import annotations

import math

import numpy as np

from .basis import Molecule

DEFAULT_SEED = 20261203


def _rand_rotation(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)],
    ])


def water_cluster(n: int, box: float, seed: int = DEFAULT_SEED, min_oo: float = 2.8,
                  max_tries: int = 200000) -> Molecule:
    rng = np.random.Generator(np.random.PCG64(seed))
    r, ang = 0.96, math.radians(104.5)
    local = np.array([[0.0, 0.0, 0.0],
                      [r * math.sin(ang / 2), 0.0, r * math.cos(ang / 2)],
                      [-r * math.sin(ang / 2), 0.0, r * math.cos(ang / 2)]])
    oxy = []
    tries = 0
    while len(oxy) < n:
        tries += 1
        if tries > max_tries:
            raise RuntimeError(f"cannot place {n} waters in a {box} A box")
        p = rng.uniform(0.0, box, size=3)
        if all(np.linalg.norm(p - q) >= min_oo for q in oxy):
            oxy.append(p)
    sym, xyz = [], []
    for p in oxy:
        R = _rand_rotation(rng)
        for k, s in enumerate(("O", "H", "H")):
            sym.append(s)
            xyz.append(p + R @ local[k])
    return Molecule.from_angstrom(sym, np.array(xyz))


def alkane(n: int, seed: int = DEFAULT_SEED, jitter: float = 0.02) -> Molecule:
    rng = np.random.Generator(np.random.PCG64(seed))
    cc, ch = 1.54, 1.09
    half = math.radians(109.4712206) / 2.0
    dx = cc * math.sin(half)
    dy = cc * math.cos(half)
    carbons = [np.array([i * dx, (i % 2) * dy, 0.0]) for i in range(n)]
    sym, xyz = [], []
    for i, c in enumerate(carbons):
        sym.append("C")
        xyz.append(c)
    # hydrogens: two per carbon out of the backbone plane, plus one extra on each end
    tet = math.radians(109.4712206)
    for i, c in enumerate(carbons):
        up = 1.0 if i % 2 == 0 else -1.0   # away from the neighbours
        # bisector pointing away from the backbone in-plane, H's tilted +/- z
        base = np.array([0.0, -up, 0.0])
        hz = math.sin(tet / 2)
        hy = math.cos(tet / 2)
        for s in (+1.0, -1.0):
            v = np.array([0.0, base[1] * hy, s * hz])
            sym.append("H")
            xyz.append(c + ch * v / np.linalg.norm(v))
    # terminal hydrogens along the chain direction
    d0 = carbons[0] - carbons[1]
    sym.append("H")
    xyz.append(carbons[0] + ch * d0 / np.linalg.norm(d0))
    d1 = carbons[-1] - carbons[-2]
    sym.append("H")
    xyz.append(carbons[-1] + ch * d1 / np.linalg.norm(d1))
    xyz = np.array(xyz) + rng.normal(scale=jitter, size=(len(xyz), 3))
    return Molecule.from_angstrom(sym, xyz)


# the workloads named by their sizes
def water4_sto3g():
    return water_cluster(4, 6.0), "STO-3G"


def water32_631gs():
    return water_cluster(32, 10.0), "6-31G*"


def c40h82_631gss():
    return alkane(40), "6-31G**"


def water12_ccpvtz():
    return water_cluster(12, 8.0), "CC-PVTZ"
