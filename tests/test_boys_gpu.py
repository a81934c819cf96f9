"""GPU test of the device Boys function F_m(T) against high-precision values.

The Fock kernels evaluate F_0..F_M in two forms: the per-lane kernels by a 7-term
Taylor step from a 0.05-spaced table below T = 36 then downward recursion, the
asymptotic form with upward recursion above it (boys_scaled_rows); the
cooperative kernels one m at a time (boys_one).  The oracle uses the same
tabulated method, so a table error common to both would pass the Fock parity
tests; this test pins the device values to mpmath directly (1F1 at 40 digits),
1e-13 relative, for m = 0..12 (ffff quartets need M = 12) and T in [0, 36) and
[36, 2000].  The reference's device Boys is src/gpu/gpu_fmt.h:5-72.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
mpmath = pytest.importorskip("mpmath")
pytestmark = pytest.mark.gpu

REL_TOL = 1e-13


def _boys_mp(m, T):
    mpmath.mp.dps = 40
    if T == 0.0:
        return 1.0 / (2 * m + 1)
    return float(mpmath.hyp1f1(m + 0.5, m + 1.5, -T) / (2 * m + 1))


def _points():
    rng = np.random.default_rng(123)
    below = np.concatenate([[0.0, 1e-12, 1e-6, 0.025, 0.0249999, 0.05, 0.075, 1.0, 17.975, 35.975, 35.999999],
                            rng.uniform(0.0, 36.0, 60)])
    above = np.concatenate([[36.0, 36.0000001, 40.0, 100.0, 777.7, 2000.0], rng.uniform(36.0, 2000.0, 20)])
    return np.concatenate([below, above])


@pytest.mark.parametrize("M", [0, 1, 2, 4, 6, 8, 10, 12])
def test_device_boys_against_mpmath(M):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from quick_b200._native import check, lib
    from quick_b200.basis import build_basis
    from quick_b200.get2e import Get2e
    from quick_b200.molecules import water_cluster
    L = lib()
    if M > 4 * L.qk_max_l():
        pytest.skip("M above the compiled maximum")
    eng = Get2e(build_basis(water_cluster(1, 3.0), "STO-3G"))
    T = _points()
    n = len(T)
    Fr = np.zeros((n, M + 1))
    F1 = np.zeros((n, M + 1))
    P = lambda a: ctypes.c_void_p(a.ctypes.data)  # noqa: E731
    check(L.qk_boys(ctypes.c_void_p(eng.h), M, P(T), n, P(Fr), P(F1)), "qk_boys")
    eng.close()
    worst = 0.0
    for i, t in enumerate(T):
        for m in range(M + 1):
            ref = _boys_mp(m, float(t))
            for got in (Fr[i, m], F1[i, m]):
                rel = abs(got - ref) / abs(ref)
                worst = max(worst, rel)
                assert rel <= REL_TOL, (M, m, float(t), got, ref, rel)
    print(f"M={M}: worst relative error {worst:.2e}")


@pytest.mark.parametrize("M", [0, 1, 2, 3, 4, 6, 8, 12])
def test_device_quick_boys_matches_oracle_restatement(M):
    """The reference-faithful mode (qk_set_boys(1)): the device copy of QUICK's
    fmt.f90 against the oracle's restatement of it, both rounding every multiply and
    add on its own.  exp() differs by an ulp between the device and the host
    library, and QUICK's upward recursion amplifies that by up to ~500 where it is
    still accurate (M = 4 at T = 0.34: 4e-13 relative) and beyond all digits where
    it is not (high M at small T); so the two copies must agree to 1e-13 relative
    plus the error of QUICK's value itself against the exact one."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from oracle import oracle as O
    from quick_b200._native import check, lib
    from quick_b200.basis import build_basis
    from quick_b200.get2e import Get2e
    from quick_b200.molecules import water_cluster
    L = lib()
    if M > 4 * L.qk_max_l():
        pytest.skip("M above the compiled maximum")
    eng = Get2e(build_basis(water_cluster(1, 3.0), "STO-3G"))
    eng.set_boys(1)
    rng = np.random.default_rng(7)
    T = np.concatenate([[1e-7, 5e-5, 1e-4, 0.05, 0.1, 0.5, 1.0, 2.0, 3.0, 4.5, 5.0, 7.0, 10.0, 12.0, 15.0, 20.0,
                         33.0, 40.0, 300.0], np.exp(rng.uniform(np.log(1e-6), np.log(100.0), 60))])
    n = len(T)
    Fr, F1 = np.zeros((n, M + 1)), np.zeros((n, M + 1))
    P = lambda a: ctypes.c_void_p(a.ctypes.data)  # noqa: E731
    check(L.qk_boys(ctypes.c_void_p(eng.h), M, P(T), n, P(Fr), P(F1)), "qk_boys")
    eng.close()
    tight = 0
    with O.quick_boys():
        for i, t in enumerate(T):
            Fq = O.boys(M, float(t))
            for m in range(M + 1):
                exact = _boys_mp(m, float(t))
                bound = 1e-13 * abs(Fq[m]) + abs(Fq[m] - exact)
                tight += abs(Fq[m] - exact) <= 1e-13 * abs(exact)
                for got in (Fr[i, m], F1[i, m]):
                    assert np.isfinite(got)
                    assert abs(got - Fq[m]) <= bound, (M, m, float(t), got, Fq[m], exact)
    assert tight > 0
