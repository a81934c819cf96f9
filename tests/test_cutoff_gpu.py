"""Cutoff changes on a live context: work lists built at a tighter cutoff give
exactly the build of fresh lists (the kernels apply the CPU get2e's two tests,
Y_ij*Y_kl > cut and Y_ij*Y_kl*DNmax > cut), and QUICK's SCF cutoff schedule
(adjust_Cutoff, src/modules/quick_method_module.f90:1107-1129) through the
eager and graph drivers."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from quick_b200.basis import build_basis  # noqa: E402
from quick_b200.molecules import water_cluster  # noqa: E402
from oracle import oracle as O  # noqa: E402


def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _density(b, seed):
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(b.nbasis, b.nbasis)) * 0.2
    return X @ X.T / b.nbasis ** 0.5


def test_lists_from_a_tighter_cutoff_give_the_fresh_build():
    _cuda()
    from quick_b200.get2e import Get2e
    b = build_basis(water_cluster(4, 6.0, seed=2), "6-31G*")
    D = _density(b, 11)
    Dt = torch.tensor(D, device="cuda")
    orc = O.Oracle(b)
    Y, cp = orc.schwarz()
    cm = orc.density_cutoff(D)
    wide = Get2e(b, integral_cutoff=1e-12, prim_limit=1e-8)
    wide.fock2e(Dt)
    listed = wide.work()["quartets"]                          # quartets on the 1e-12 lists
    for cut, prim in [(1e-7, 1e-8), (1e-9, 1e-9), (1e-10, 1e-11)]:
        wide.set_cutoffs(cut, prim)
        got = wide.fock2e(Dt)
        assert wide.work()["quartets"] == listed              # the 1e-12 lists were kept
        fresh = Get2e(b, integral_cutoff=cut, prim_limit=prim)
        want = fresh.fock2e(Dt)
        assert fresh.work()["quartets"] < listed
        assert torch.equal(got, want), cut                    # same quartet set, int64 sums
        ref, _ = orc.get2e(D, cm, Y, cp, cut, prim)
        assert np.abs(got.cpu().numpy() - ref).max() <= 1e-9, cut
        fresh.close()
    # tightening below the lists rebuilds them
    wide.set_cutoffs(1e-13, 1e-14)
    got = wide.fock2e(Dt)
    assert wide.work()["quartets"] > listed
    ref, _ = orc.get2e(D, cm, Y, cp, 1e-13, 1e-14)
    assert np.abs(got.cpu().numpy() - ref).max() <= 1e-9
    wide.close()


def test_noalloc_build_accepts_lists_from_a_tighter_cutoff():
    _cuda()
    import ctypes
    from quick_b200._native import check, lib
    from quick_b200.get2e import Get2e
    b = build_basis(water_cluster(3, 6.0, seed=6), "6-31G*")
    Dt = torch.tensor(_density(b, 3), device="cuda")
    eng = Get2e(b, integral_cutoff=1e-11, prim_limit=1e-12)
    eng.prepare()
    eng.set_cutoffs(1e-8, 1e-9)
    want = eng.fock2e(Dt)
    o = torch.zeros_like(Dt)
    s = torch.cuda.current_stream()
    check(lib().qk_fock2e_device_noalloc(eng.h, ctypes.c_void_p(Dt.data_ptr()), None, ctypes.c_void_p(o.data_ptr()),
                                         ctypes.c_void_p(s.cuda_stream)), "qk_fock2e_device_noalloc")
    torch.cuda.synchronize()
    assert torch.equal(o, want)
    eng.close()


def test_adaptive_cutoff_scf_eager_and_graph():
    _cuda()
    from quick_b200.scf import RHF, GraphSCF
    b = build_basis(water_cluster(5, 6.5, seed=5), "6-31G*")
    tight = RHF(b, integral_cutoff=1e-11, prim_limit=1e-11).run(denserms=1e-7)
    rhf = RHF(b, integral_cutoff=1e-7, prim_limit=1e-8)
    got = rhf.run(denserms=1e-7, adaptive_cutoff=True)
    assert tight["converged"] and got["converged"]
    cuts = [c for _, c, _ in got["cutoff_changes"]]
    assert cuts and cuts == sorted(cuts, reverse=True) and cuts[-1] <= 1e-10, got["cutoff_changes"]
    assert (rhf.eng.integral_cutoff, rhf.eng.prim_limit) == (1e-7, 1e-8)     # restored
    # QUICK keeps the incremental builds across a change, so the early, looser
    # builds stay in F: a few 1e-7 Eh (the oracle's emulation of the same
    # schedule lands 0.05-0.5 uEh from the tight solve on such clusters)
    assert abs(got["E"] - tight["E"]) <= 2e-6, (got["E"], tight["E"])
    g = GraphSCF(RHF(b, integral_cutoff=1e-7, prim_limit=1e-8)).run(denserms=1e-7, adaptive_cutoff=True)
    assert g["converged"] and g["graph"] and g["recaptures"] >= 1
    assert g["cutoff_changes"] and g["cutoff_changes"][-1][1] <= 1e-10
    assert abs(g["E"] - tight["E"]) <= 2e-6, (g["E"], tight["E"])
