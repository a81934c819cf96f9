"""GPU parity at the benchmark sizes: the CUDA Fock build and SCF against the CPU
oracle on the named workloads themselves, not only on small clusters.

* 32 H2O / 6-31G* (608 functions, the benchmark workload): G on the
  core-Hamiltonian density and on a random density, max |dG| <= 1e-9 Eh; the RHF
  energy through the GPU Fock build, the eager GPU SCF and the graph-captured GPU
  SCF, each within 1e-7 Eh of the oracle's SCF.
* C40H82 / 6-31G** (1010 functions) and 12 H2O / cc-pVTZ (780 functions, f
  shells): one G build each, max |dG| <= 1e-9 Eh.
* QUICK's own CUDA get2e (built from the reference sources by
  oracle/Makefile.refgpu, run through its C entry points): its G against the
  oracle and against this library's on 4 H2O / STO-3G and 32 H2O / 6-31G*.

Reference semantics: get_cshell_eri / cshell / iclass_cshell,
src/modules/include/eri.fh:161-1058.  The oracle runs on all host threads.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from quick_b200.basis import build_basis  # noqa: E402
from quick_b200 import molecules as M  # noqa: E402
from oracle import oracle as O  # noqa: E402

FOCK_TOL = 1e-9
ENERGY_TOL = 1e-7
CUT, PRIM = 1e-10, 1e-11


def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _core_density(b):
    S, T, V = O.oei(b)
    X = O.orthogonalizer(S)
    e, C = np.linalg.eigh(X.T @ (T + V) @ X)
    C = X @ C[:, :b.mol.nelec // 2]
    return 2.0 * C @ C.T


def _random_density(n, seed):
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(n, n)) * 0.15
    return X @ X.T / n ** 0.5


_CACHE = {}


def _setup(name):
    if name not in _CACHE:
        mol, bas = {"w32": M.water32_631gs, "c40": M.c40h82_631gss, "w12": M.water12_ccpvtz,
                    "w4": M.water4_sto3g}[name]()
        b = build_basis(mol, bas)
        orc = O.Oracle(b)
        _CACHE[name] = (b, orc, orc.schwarz())
    return _CACHE[name]


def _gpu_fock(b, D, Y, cp, cut=CUT, prim=PRIM, boys_mode=0):
    from quick_b200.get2e import Get2e
    eng = Get2e(b, integral_cutoff=cut, prim_limit=prim, schwarz=(Y, cp))
    eng.set_boys(boys_mode)
    G = eng.fock2e(torch.tensor(D, device="cuda")).cpu().numpy()
    eng.close()
    return G


@pytest.mark.parametrize("name,density", [("w32", "core"), ("w32", "random"), ("c40", "random"),
                                          ("w12", "random")])
def test_fock_matches_oracle_at_workload_size(name, density):
    _cuda()
    b, orc, (Y, cp) = _setup(name)
    D = _core_density(b) if density == "core" else _random_density(b.nbasis, 17)
    cm = orc.density_cutoff(D)
    G_ref, _ = orc.get2e(D, cm, Y, cp, CUT, PRIM)
    G = _gpu_fock(b, D, Y, cp)
    err = float(np.abs(G - G_ref).max())
    assert err <= FOCK_TOL, f"{name}/{density}: max |dG| = {err:.3e}"
    assert np.array_equal(G, G.T)


@pytest.fixture(scope="module")
def w32_scf():
    """The oracle's RHF on 32 H2O / 6-31G* (SAD start, cutoff 1e-11) and the same
    SCF with the GPU Fock build in its place."""
    _cuda()
    from quick_b200.get2e import Get2e
    from quick_b200.guess import sad_density
    b, orc, (Y, cp) = _setup("w32")
    D0 = sad_density(b)
    D0 = D0.cpu().numpy() if hasattr(D0, "cpu") else np.asarray(D0)
    ref = O.rhf(b, integral_cutoff=1e-11, prim_limit=1e-12, conv=1e-8, guess=D0)
    eng = Get2e(b, integral_cutoff=1e-11, prim_limit=1e-12, schwarz=(Y, cp))

    def fb(D, cm):
        return eng.fock2e(torch.tensor(D, device="cuda"), cutmat=torch.tensor(cm, device="cuda")).cpu().numpy()

    got = O.rhf(b, integral_cutoff=1e-11, prim_limit=1e-12, conv=1e-8, guess=D0, fock_builder=fb)
    eng.close()
    return b, ref, got


def test_w32_scf_energy_through_gpu_fock_build(w32_scf):
    b, ref, got = w32_scf
    assert abs(got["E"] - ref["E"]) <= ENERGY_TOL, (got["E"], ref["E"])


@pytest.mark.parametrize("driver", ["eager", "graph"])
def test_w32_gpu_scf_drivers_match_oracle_energy(w32_scf, driver):
    from quick_b200.scf import RHF, GraphSCF
    b, ref, _ = w32_scf
    rhf = RHF(b, integral_cutoff=1e-11, prim_limit=1e-12)
    if driver == "eager":
        r = rhf.run(denserms=1e-8, guess="sad")
    else:
        r = GraphSCF(rhf).run(denserms=1e-8, guess="sad")
    rhf.eng.close()
    assert r["converged"]
    assert abs(r["E"] - ref["E"]) <= ENERGY_TOL, (driver, r["E"], ref["E"])


# ---------------------------------------------------------------- QUICK's own GPU get2e
def _refgpu():
    from oracle import refgpu
    if not refgpu.available():
        pytest.skip("QUICK's GPU get2e harness is not built (oracle/Makefile.refgpu)")
    return refgpu


@pytest.mark.parametrize("name", ["w4", "w32"])
def test_reference_gpu_get2e_matches_oracle_and_ours(name):
    """QUICK's own GPU get2e against the oracle and this library.

    The oracle is run the way that GPU path computes: QUICK's own Boys function
    (src/subs/fmt.f90, whose device copy is src/gpu/gpu_fmt.h) and its two extra
    screens (shell pairs with Y > 1e-10 only, src/gpu/cuda/gpu.cu:929-1030;
    integrals with |Y| <= integralCutoff not digested,
    src/gpu/gpu_get2e_subs.h:389).  Measured at cutoff 1e-10: 2.6e-8 (4 H2O) and
    2.2e-6 (32 H2O), all of it in rows of s functions; the Boys function accounts
    for 2.6e-8 and 1.1e-6 of the difference between the reference's GPU result
    and the accurate oracle (5.2e-8 and 2.3e-6).  The bound is 5e-6.  This
    library with QUICK's Boys function at the order the GPU path evaluates it
    (qk_set_boys(2), the split s/p class's M) reproduces that path's G to 2.5e-9
    and 2.3e-8 Eh."""
    _cuda()
    refgpu = _refgpu()
    b, orc, (Y, cp) = _setup(name)
    D = _core_density(b)
    cm = orc.density_cutoff(D)
    G_orc, _ = orc.get2e(D, cm, Y, cp, CUT, PRIM)
    with O.quick_boys():
        G_orc_q, _ = orc.get2e(D, cm, Y, cp, CUT, PRIM, gpu_screens=True)
    G_ref, info = refgpu.run(b, D, cm, Y, cp, CUT, PRIM, steps=2, warmup=1)
    G = _gpu_fock(b, D, Y, cp)
    G_gpu_order = _gpu_fock(b, D, Y, cp, boys_mode=2)
    e_mine = float(np.abs(G_gpu_order - G_ref).max())
    e_q = float(np.abs(G_ref - G_orc_q).max())
    e_plain = float(np.abs(G_ref - G_orc).max())
    e_ours = float(np.abs(G - G_orc).max())
    print(f"{name}: |G_refgpu - G_oracle(QUICK Boys, GPU screens)| = {e_q:.3e}, |G_refgpu - G_oracle| = "
          f"{e_plain:.3e}, |G_ours - G_oracle| = {e_ours:.3e}, |G_ours(GPU-order QUICK Boys) - G_refgpu| = "
          f"{e_mine:.3e}, {info}")
    assert info["bit_identical_repeat"]
    # QUICK's Boys function at the order its GPU path uses (qk_set_boys(2)) accounts
    # for all but 2.5e-9 (4 H2O) and 2.3e-8 Eh (32 H2O) of that path's result
    assert e_mine <= 1e-7, e_mine
    assert e_q <= 5e-6, e_q
    assert e_plain <= 5e-6, e_plain
    assert e_ours <= FOCK_TOL, e_ours
