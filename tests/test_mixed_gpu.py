"""GPU tests of the mixed FP32/FP64 form (quartets with a small Schwarz bound
product evaluate the vertical recursion in FP32).  Tolerances: the Fock matrix
stays within 1e-7 Eh of the FP64 build, and the SCF energy within 1 uEh."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from quick_b200.basis import build_basis  # noqa: E402
from quick_b200.molecules import water_cluster  # noqa: E402


def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


@pytest.mark.parametrize("bound", [1e-6, 1e-5, 1e-4])
def test_mixed_fock_close_to_fp64(bound):
    _cuda()
    from quick_b200.get2e import Get2e
    b = build_basis(water_cluster(6, 7.0, seed=5), "6-31G*")
    eng = Get2e(b, integral_cutoff=1e-10, prim_limit=1e-11)
    rng = np.random.default_rng(4)
    X = rng.normal(size=(b.nbasis, b.nbasis)) * 0.15
    D = torch.tensor(X @ X.T / b.nbasis ** 0.5, device="cuda")
    G64 = eng.fock2e(D).cpu().numpy()
    eng.set_precision(bound)
    G32 = eng.fock2e(D).cpu().numpy()
    assert eng.fp32_quartets() > 0
    err = float(np.abs(G32 - G64).max())
    assert err <= 1e-7, err
    G32b = eng.fock2e(D).cpu().numpy()
    assert G32.tobytes() == G32b.tobytes()        # still bit-reproducible
    eng.set_precision(0.0)
    assert eng.fock2e(D).cpu().numpy().tobytes() == G64.tobytes()
    eng.close()


def test_mixed_scf_energy_within_1_microhartree():
    _cuda()
    from quick_b200.scf import RHF
    b = build_basis(water_cluster(8, 8.0, seed=9), "6-31G*")
    ref = RHF(b, integral_cutoff=1e-10).run(denserms=1e-7)
    rhf = RHF(b, integral_cutoff=1e-10)
    rhf.eng.set_precision(1e-5)
    got = rhf.run(denserms=1e-7)
    assert ref["converged"] and got["converged"]
    assert abs(got["E"] - ref["E"]) <= 1e-6, (got["E"], ref["E"])


# ------------------------------------------------ error against the FP64 oracle
def test_mixed_fock_error_against_oracle():
    """The mixed form's G against the CPU oracle (the FP64 reference restatement),
    same density and screens: max |dG| <= 1e-7 Eh, and the FP64 build <= 1e-9."""
    _cuda()
    from oracle import oracle as O
    from quick_b200.get2e import Get2e
    b = build_basis(water_cluster(6, 7.0, seed=5), "6-31G*")
    orc = O.Oracle(b)
    Y, cp = orc.schwarz()
    rng = np.random.default_rng(4)
    X = rng.normal(size=(b.nbasis, b.nbasis)) * 0.15
    Dn = X @ X.T / b.nbasis ** 0.5
    G_orc, _ = orc.get2e(Dn, orc.density_cutoff(Dn), Y, cp, 1e-10, 1e-11)
    eng = Get2e(b, integral_cutoff=1e-10, prim_limit=1e-11, schwarz=(Y, cp))
    D = torch.tensor(Dn, device="cuda")
    assert float(np.abs(eng.fock2e(D).cpu().numpy() - G_orc).max()) <= 1e-9
    for bound in (1e-6, 1e-5, 1e-4):
        eng.set_precision(bound)
        err = float(np.abs(eng.fock2e(D).cpu().numpy() - G_orc).max())
        assert err <= 1e-7, (bound, err)
    eng.close()


def test_mixed_scf_energy_against_oracle():
    """The mixed-form SCF energy against the oracle's FP64 SCF: |dE| <= 1 uEh."""
    _cuda()
    from oracle import oracle as O
    from quick_b200.guess import sad_density
    from quick_b200.scf import RHF
    b = build_basis(water_cluster(8, 8.0, seed=9), "6-31G*")
    ref = O.rhf(b, integral_cutoff=1e-11, prim_limit=1e-12, conv=1e-8, guess=sad_density(b))
    rhf = RHF(b, integral_cutoff=1e-11, prim_limit=1e-12)
    rhf.eng.set_precision(1e-5)
    got = rhf.run(denserms=1e-8)
    assert got["converged"]
    assert abs(got["E"] - ref["E"]) <= 1e-6, (got["E"], ref["E"])
    rhf.eng.close()
