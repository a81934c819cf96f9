"""GPU tests of the graph-captured SCF iteration (GraphSCF) and its device-side
pieces: the DIIS solve kernel and the SP2 density projection."""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from quick_b200.basis import build_basis  # noqa: E402
from quick_b200.molecules import water_cluster  # noqa: E402


def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _solve(A, b):
    from quick_b200._native import lib
    n = A.shape[0]
    Ad = torch.tensor(A, device="cuda")
    bd = torch.tensor(b, device="cuda")
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    ok = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = torch.cuda.current_stream()
    assert lib().qk_small_solve(ctypes.c_void_p(Ad.data_ptr()), ctypes.c_void_p(bd.data_ptr()), n,
                                ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(ok.data_ptr()),
                                ctypes.c_void_p(st.cuda_stream)) == 0
    return x.cpu().numpy(), int(ok.item())


@pytest.mark.parametrize("n", [1, 2, 11, 33, 64])
def test_small_solve_matches_numpy(n):
    _cuda()
    rng = np.random.default_rng(n)
    A = rng.normal(size=(n, n)) + n * np.eye(n) * 0.1
    b = rng.normal(size=n)
    x, ok = _solve(A, b)
    assert ok == 1
    assert np.allclose(x, np.linalg.solve(A, b), rtol=1e-10, atol=1e-12)


def test_small_solve_diis_shape_and_singular():
    _cuda()
    # the DIIS matrix: zero corner, -1 border -> needs pivoting
    rng = np.random.default_rng(1)
    E = rng.normal(size=(5, 40))
    B = -np.ones((6, 6))
    B[:5, :5] = E @ E.T
    B[5, 5] = 0.0
    rhs = np.zeros(6)
    rhs[5] = -1.0
    x, ok = _solve(B, rhs)
    assert ok == 1 and abs(x[:5].sum() - 1.0) < 1e-12
    assert np.allclose(x, np.linalg.solve(B, rhs), rtol=1e-9, atol=1e-12)
    x, ok = _solve(np.zeros((4, 4)), np.ones(4))
    assert ok == 0 and not x.any()


@pytest.mark.parametrize("n,nocc", [(1, 0.0), (37, 5.0), (37, 30.0), (300, 41.0)])
def test_sp2_step_matches_formula(n, nocc):
    """qk_sp2_step against the step written out in torch, both branches."""
    _cuda()
    from quick_b200._native import check, lib
    g = torch.Generator().manual_seed(n)
    A = torch.randn(n, n, generator=g, dtype=torch.float64)
    Y = ((A + A.T) / (4.0 * n ** 0.5) + 0.5 * torch.eye(n, dtype=torch.float64)).cuda()
    Y2 = Y @ Y
    out = torch.full_like(Y, float("nan"))
    s = torch.cuda.current_stream()
    vp = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    check(lib().qk_sp2_step(vp(Y), vp(Y2), vp(out), n, nocc, ctypes.c_void_p(s.cuda_stream)), "qk_sp2_step")
    t0, t1 = float(torch.trace(Y)), float(torch.trace(Y2))
    want = Y2 if abs(t1 - nocc) < abs(2.0 * t0 - t1 - nocc) else 2.0 * Y - Y2
    assert torch.equal(out, want)
    assert lib().qk_sp2_step(vp(Y), vp(Y2), vp(Y), n, nocc, ctypes.c_void_p(s.cuda_stream)) != 0   # aliasing refused


@pytest.mark.parametrize("n,nocc,steps", [(37, 5.0, 0), (37, 5.0, 7), (37, 5.0, None), (300, 41.0, None),
                                           (608, 160.0, None)])
def test_sp2_run_equals_stepwise_loop(n, nocc, steps):
    """qk_sp2_run against the same steps taken one at a time from Python (torch's
    GEMM and qk_sp2_step): the same matrix to 1e-12 (both GEMMs are cuBLAS's, run
    through different handles), result in Ya after an even step count and Yb after
    an odd one; with the SCF's step count (sp2_steps) the purified matrix is
    idempotent with trace nocc."""
    _cuda()
    from quick_b200._native import check, lib
    from quick_b200.scf import sp2_steps
    g = torch.Generator().manual_seed(n)
    A = torch.randn(n, n, generator=g, dtype=torch.float64)
    _, U = torch.linalg.eigh((A + A.T) / 2.0)
    w = torch.linspace(-2.0, 1.0, n, dtype=torch.float64)          # a clean gap at every nocc
    F = (U * w) @ U.T
    d = torch.diagonal(F)
    rad = F.abs().sum(dim=1) - d.abs()
    emin, emax = float((d - rad).min()), float((d + rad).max())
    Y0 = ((emax * torch.eye(n, dtype=torch.float64) - F) / (emax - emin)).cuda()
    converge = steps is None
    if converge:
        steps = sp2_steps(w.numpy(), int(nocc), emax - emin)
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    vp = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    Ya, Yb, Y2 = Y0.clone(), torch.zeros_like(Y0), torch.zeros_like(Y0)
    check(lib().qk_sp2_run(vp(Ya), vp(Yb), vp(Y2), n, nocc, steps, s), "qk_sp2_run")
    got = Ya if steps % 2 == 0 else Yb
    cur, nxt, Z2 = Y0.clone(), torch.zeros_like(Y0), torch.zeros_like(Y0)
    for _ in range(steps):
        torch.mm(cur, cur, out=Z2)
        check(lib().qk_sp2_step(vp(cur), vp(Z2), vp(nxt), n, nocc, s), "qk_sp2_step")
        cur, nxt = nxt, cur
    assert float((got - cur).abs().max()) <= 1e-12
    if converge:
        assert abs(float(torch.trace(got)) - nocc) < 1e-8
        assert float((got @ got - got).abs().max()) < 1e-8
    assert lib().qk_sp2_run(vp(Ya), vp(Ya), vp(Y2), n, nocc, steps, s) != 0   # aliasing refused


def test_sp2_projector_equals_diagonalisation():
    _cuda()
    from quick_b200.scf import RHF, GraphSCF, gershgorin_range, sp2_steps
    b = build_basis(water_cluster(3, 6.0, seed=2), "6-31G*")
    rhf = RHF(b, integral_cutoff=1e-10)
    F = rhf.run(denserms=1e-6)["F"]           # a Fock matrix with the SCF's HOMO-LUMO gap
    e, C = torch.linalg.eigh(rhf.X.T @ F @ rhf.X)
    Co = rhf.X @ C[:, : rhf.nocc]
    D_ref = 2.0 * Co @ Co.T
    ev = e.cpu().numpy()
    g = GraphSCF(rhf, sp2=sp2_steps(ev, rhf.nocc, gershgorin_range(rhf.X.T @ F @ rhf.X)))
    D = g._density(F)
    err = float(torch.abs(D - D_ref).max())
    assert abs(float(g.out[3])) < 1e-10
    assert err < 1e-10, (err, g.sp2, ev[rhf.nocc - 1], ev[rhf.nocc], ev[0], ev[-1])


@pytest.mark.parametrize("bas,nw", [("STO-3G", 4), ("6-31G*", 5)])
def test_graph_scf_matches_eager_and_eigh(bas, nw):
    _cuda()
    from quick_b200.scf import RHF, GraphSCF
    b = build_basis(water_cluster(nw, 6.5, seed=nw), bas)
    ref = RHF(b, integral_cutoff=1e-10).run(denserms=1e-7)
    eager = GraphSCF(RHF(b, integral_cutoff=1e-10)).run(denserms=1e-7, graph=False)
    graph = GraphSCF(RHF(b, integral_cutoff=1e-10)).run(denserms=1e-7, graph=True)
    assert ref["converged"] and eager["converged"] and graph["converged"] and graph["graph"]
    # same kernels, same numbers
    assert graph["niter"] == eager["niter"]
    assert graph["E"] == eager["E"]
    assert torch.equal(graph["D"], eager["D"])
    # SP2 + fixed-slot DIIS against diagonalisation + growing DIIS
    assert abs(graph["E"] - ref["E"]) < 1e-9, (graph["E"], ref["E"])
    assert abs(graph["niter"] - ref["niter"]) <= 2


def test_graph_scf_mixed_precision_within_1_microhartree():
    _cuda()
    from quick_b200.scf import RHF, GraphSCF
    b = build_basis(water_cluster(6, 7.0, seed=3), "6-31G*")
    ref = GraphSCF(RHF(b, integral_cutoff=1e-10)).run(denserms=1e-7)
    rhf = RHF(b, integral_cutoff=1e-10)
    rhf.eng.set_precision(1e-5)
    got = GraphSCF(rhf).run(denserms=1e-7)
    assert got["converged"] and abs(got["E"] - ref["E"]) <= 1e-6
