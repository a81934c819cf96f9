"""GPU test of the allocation-free Fock build, qk_fock2e_device_noalloc.

Some callers of this library cannot allocate device memory when they need a
Fock build: a host program that fixes its GPU memory pool at start-up, or code
that must not call cudaMalloc/cudaFree because those synchronise the whole
device.  The allocation-free entry point serves them: its per-build scratch
lives in a fixed array inside the library, and the caller passes only the
density and the output buffer.

The test drives that entry point through the C ABI and checks its result
against the ordinary entry point (qk_fock2e_device) on the same density, within
the Fock tolerance of the other GPU tests, on two calls in a row (the second
call reuses the scratch that the first one left behind).  This file is named so
that pytest collects it last; it also passes when run alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

FOCK_TOL = 1e-9


def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _random_density(n, seed):
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(n, n)) * 0.15
    return X @ X.T / n ** 0.5


def test_noalloc_matches_allocating_entry_point_twice():
    _cuda()
    from quick_b200 import _native
    from quick_b200.basis import build_basis
    from quick_b200.get2e import Get2e
    from quick_b200.molecules import water_cluster

    L = _native.lib()
    b = build_basis(water_cluster(3, 6.0, seed=11), "6-31G*")
    eng = Get2e(b, integral_cutoff=1e-10, prim_limit=1e-11)
    h = ctypes.c_void_p(eng.h)
    n = b.nbasis
    stream = torch.cuda.current_stream()
    vp = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731

    D = torch.tensor(_random_density(n, 21), device="cuda")
    # before any ordinary build the pair tables do not exist yet: a clear refusal
    o = torch.zeros((n, n), dtype=torch.float64, device="cuda")
    assert L.qk_fock2e_device_noalloc(h, vp(D), None, vp(o), ctypes.c_void_p(stream.cuda_stream)) == 102

    ref = eng.fock2e(D).cpu().numpy()          # ordinary entry point (builds the tables)
    for call in range(2):
        o = torch.zeros((n, n), dtype=torch.float64, device="cuda")
        st = L.qk_fock2e_device_noalloc(h, vp(D), None, vp(o), ctypes.c_void_p(stream.cuda_stream))
        assert st == 0, (call, st)
        got = o.cpu().numpy()
        err = float(np.abs(got - ref).max())
        assert err <= FOCK_TOL, (call, err)

    # a caller-provided density screen goes through the same path
    cm = eng.density_cutoff(D)
    o = torch.zeros((n, n), dtype=torch.float64, device="cuda")
    assert L.qk_fock2e_device_noalloc(h, vp(D), vp(cm), vp(o), ctypes.c_void_p(stream.cuda_stream)) == 0
    assert float(np.abs(o.cpu().numpy() - ref).max()) <= FOCK_TOL
    eng.close()


def _noalloc(L, eng, D, o, cm=None):
    s = torch.cuda.current_stream()
    vp = lambda t: ctypes.c_void_p(t.data_ptr()) if t is not None else None  # noqa: E731
    st = L.qk_fock2e_device_noalloc(ctypes.c_void_p(eng.h), vp(D), vp(cm), vp(o), ctypes.c_void_p(s.cuda_stream))
    torch.cuda.synchronize()
    return st


def test_noalloc_refuses_stale_lists_and_follows_precision_and_streams():
    """Any change that makes the ordinary entry point rebuild its work lists (a
    tighter cutoff, another FP32 bound) is refused with 102 by the allocation-free
    one, which cannot build them; after one ordinary build it matches again,
    mixed precision included.  It follows the launch shape of qk_set_streams and
    reports its own work counts through qk_last_work."""
    _cuda()
    from quick_b200 import _native
    from quick_b200.basis import build_basis
    from quick_b200.get2e import Get2e
    from quick_b200.molecules import water_cluster

    L = _native.lib()
    b = build_basis(water_cluster(3, 6.0, seed=11), "6-31G*")
    n = b.nbasis
    eng = Get2e(b, integral_cutoff=1e-9, prim_limit=1e-10)
    D = torch.tensor(_random_density(n, 23), device="cuda")
    z = lambda: torch.zeros((n, n), dtype=torch.float64, device="cuda")  # noqa: E731

    eng.fock2e(D)
    eng.set_cutoffs(1e-11, 1e-12)                 # tighter: the lists must be rebuilt
    assert _noalloc(L, eng, D, z()) == 102
    ref = eng.fock2e(D).cpu().numpy()
    o = z()
    assert _noalloc(L, eng, D, o) == 0
    assert float(np.abs(o.cpu().numpy() - ref).max()) <= FOCK_TOL

    eng.set_precision(1e-5)                       # another FP32 bound: another work split
    assert _noalloc(L, eng, D, z()) == 102
    ref32 = eng.fock2e(D).cpu().numpy()
    assert eng.fp32_quartets() > 0
    for _ in range(2):
        o = z()
        assert _noalloc(L, eng, D, o) == 0
        assert o.cpu().numpy().tobytes() == ref32.tobytes()   # same items, same int64 sums
    eng.set_precision(0.0)
    assert _noalloc(L, eng, D, z()) == 102
    eng.fock2e(D)

    eng.set_streams(0)                            # one class after another
    o = z()
    assert _noalloc(L, eng, D, o) == 0
    assert o.cpu().numpy().tobytes() == ref.tobytes()
    want = eng.work()
    eng.fock2e(D)                                 # ordinary build: same counts
    got = eng.work()
    assert want["quartets"] == got["quartets"] > 0 and want["prim_quartets"] == got["prim_quartets"]

    eng.set_shard(0, 2)                           # a sharded context never finalises a part
    assert _noalloc(L, eng, D, z()) == 101
    eng.close()


def test_noalloc_size_limits():
    """Beyond the fixed scratch: nbasis > 1024 is refused (101) before anything
    runs; nshell > 512 is refused without a caller density screen and accepted
    with one."""
    _cuda()
    from quick_b200 import _native
    from quick_b200.basis import build_basis
    from quick_b200.get2e import Get2e
    from quick_b200.molecules import water_cluster

    L = _native.lib()
    big = build_basis(water_cluster(55, 13.0, seed=2), "6-31G*")     # 1045 functions
    assert big.nbasis > 1024
    eng = Get2e(big, integral_cutoff=1e-9, prim_limit=1e-10)
    n = big.nbasis
    D = torch.zeros((n, n), dtype=torch.float64, device="cuda")
    assert _noalloc(L, eng, D, torch.zeros_like(D)) == 101
    eng.close()

    many = build_basis(water_cluster(130, 17.0, seed=2), "STO-3G")   # 520 shells, 910 functions
    assert many.nshell > 512 and many.nbasis <= 1024
    eng = Get2e(many, integral_cutoff=1e-9, prim_limit=1e-10)
    n = many.nbasis
    D = torch.tensor(_random_density(n, 5), device="cuda")
    ref = eng.fock2e(D).cpu().numpy()
    assert _noalloc(L, eng, D, torch.zeros_like(D)) == 101
    cm = eng.density_cutoff(D)
    o = torch.zeros_like(D)
    assert _noalloc(L, eng, D, o, cm) == 0
    assert float(np.abs(o.cpu().numpy() - ref).max()) <= FOCK_TOL
    eng.close()
