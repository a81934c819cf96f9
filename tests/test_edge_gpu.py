"""GPU edge cases of the Fock build and its boundary: empty work, single atoms,
charged molecules, extreme cutoffs, shells outside the compiled range, and bad
arguments (the statuses of the C ABI)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from quick_b200.basis import Molecule, build_basis  # noqa: E402
from quick_b200.molecules import water_cluster  # noqa: E402
from oracle import oracle as O  # noqa: E402


def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _rand_density(n, seed):
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(n, n)) * 0.15
    return X @ X.T / n ** 0.5


def test_zero_density_gives_exact_zero():
    """Every quartet fails the density screen: no work, G exactly 0."""
    _cuda()
    from quick_b200.get2e import Get2e
    b = build_basis(water_cluster(3, 6.0, seed=1), "6-31G*")
    eng = Get2e(b, integral_cutoff=1e-10, prim_limit=1e-11)
    G = eng.fock2e(torch.zeros((b.nbasis, b.nbasis), dtype=torch.float64, device="cuda"))
    assert not bool(G.any())
    assert eng.work()["quartets"] > 0          # quartets were listed, none computed
    eng.close()


@pytest.mark.parametrize("sym,bas", [("O", "6-31G*"), ("H", "STO-3G"), ("C", "CC-PVTZ")])
def test_single_atom_matches_oracle(sym, bas):
    _cuda()
    from quick_b200.get2e import Get2e
    b = build_basis(Molecule.from_angstrom([sym], [[0.1, -0.2, 0.3]]), bas)
    orc = O.Oracle(b)
    Y, cp = orc.schwarz()
    D = _rand_density(b.nbasis, 7)
    cm = orc.density_cutoff(D)
    ref, _ = orc.get2e(D, cm, Y, cp, 1e-10, 1e-11)
    eng = Get2e(b, integral_cutoff=1e-10, prim_limit=1e-11)
    G = eng.fock2e(torch.tensor(D, device="cuda"), cutmat=torch.tensor(cm, device="cuda")).cpu().numpy()
    assert np.abs(G - ref).max() <= 1e-9
    eng.close()


@pytest.mark.parametrize("cut", [1e-3, 1e-6, 1e-13])
def test_extreme_cutoffs_match_oracle(cut):
    _cuda()
    from quick_b200.get2e import Get2e
    b = build_basis(water_cluster(2, 5.0, seed=4), "6-31G**")
    orc = O.Oracle(b)
    Y, cp = orc.schwarz()
    D = _rand_density(b.nbasis, 9)
    cm = orc.density_cutoff(D)
    ref, _ = orc.get2e(D, cm, Y, cp, cut, 0.1 * cut)
    eng = Get2e(b, integral_cutoff=cut, prim_limit=0.1 * cut)
    G = eng.fock2e(torch.tensor(D, device="cuda"), cutmat=torch.tensor(cm, device="cuda")).cpu().numpy()
    assert np.abs(G - ref).max() <= 1e-9, cut
    eng.close()


def test_charged_molecule_scf_matches_oracle():
    """H3O+ (10 electrons): the charge enters the electron count, not the build."""
    _cuda()
    from quick_b200.get2e import Get2e
    mol = Molecule.from_angstrom(["O", "H", "H", "H"], [[0.0, 0.0, 0.1], [0.95, 0.0, -0.2], [-0.47, 0.82, -0.2],
                                                       [-0.47, -0.82, -0.2]], charge=1)
    b = build_basis(mol, "6-31G*")
    assert mol.nelec == 10
    ref = O.rhf(b, guess="gwh")
    eng = Get2e(b, integral_cutoff=1e-11, prim_limit=1e-12)

    def fb(D, cm):
        return eng.fock2e(torch.tensor(D, device="cuda"), cutmat=torch.tensor(cm, device="cuda")).cpu().numpy()

    got = O.rhf(b, guess="gwh", fock_builder=fb)
    assert abs(got["E"] - ref["E"]) <= 1e-7
    from quick_b200.scf import RHF
    r = RHF(b, integral_cutoff=1e-11).run(denserms=1e-8)
    assert r["converged"] and abs(r["E"] - ref["E"]) <= 1e-6
    eng.close()


def test_shells_above_f_are_rejected():
    _cuda()
    from quick_b200._native import QuickError
    from quick_b200.get2e import Get2e
    b = build_basis(water_cluster(1, 5.0, seed=1), "STO-3G")
    b.qstart = b.qstart.copy()
    b.qfinal = b.qfinal.copy()
    b.qstart[0] = b.qfinal[0] = 4                 # a g shell, as the reference's ierr 37
    with pytest.raises(QuickError) as e:
        Get2e(b)
    assert e.value.status == 105                  # QK_ERR_UNSUPPORTED


def test_bad_arguments_are_rejected():
    _cuda()
    from quick_b200._native import QuickError
    from quick_b200.get2e import Get2e, Get2eBatch
    b = build_basis(water_cluster(1, 5.0, seed=1), "STO-3G")
    eng = Get2e(b)
    with pytest.raises(QuickError):
        eng.set_precision(-1.0)
    with pytest.raises(QuickError):
        eng.set_streams(9)
    with pytest.raises(ValueError):
        eng.fock2e(torch.zeros((b.nbasis + 1, b.nbasis + 1), dtype=torch.float64, device="cuda"))
    bt = Get2eBatch()
    assert bt.fock2e([], []) == []
    bt.close()
    eng.close()
