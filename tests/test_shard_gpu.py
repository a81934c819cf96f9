"""One Fock build split into shards (Get2e.set_shard / accumulate, the GPU form of
the reference's MPI split of the work, src/mpi_setup.f90:295-354): the shards'
int64 accumulators summed and finalised once equal the one-context build bit for
bit.  The shards run one after another on one GPU here; across GPUs the sum is
one integer all-reduce (tests/test_multirank.py checks that collective on CPU)."""
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


@pytest.mark.parametrize("bas,count", [("6-31G*", 2), ("6-31G*", 3), ("CC-PVTZ", 4)])
def test_shards_sum_to_the_full_build(bas, count):
    _cuda()
    from quick_b200._native import check, lib
    from quick_b200.get2e import Get2e
    b = build_basis(water_cluster(3, 6.0, seed=3), bas)
    n = b.nbasis
    rng = np.random.default_rng(5)
    X = rng.normal(size=(n, n)) * 0.2
    Dt = torch.tensor(X @ X.T / n ** 0.5, device="cuda")
    ref = Get2e(b, integral_cutoff=1e-10, prim_limit=1e-11)
    want = ref.fock2e(Dt)
    listed = ref.work()["quartets"]
    A = torch.zeros((n, n), dtype=torch.int64, device="cuda")
    got_listed = 0
    for r in range(count):
        e = Get2e(b, integral_cutoff=1e-10, prim_limit=1e-11)
        e.set_shard(r, count)
        e.accumulate(Dt, A)
        got_listed += e.work()["quartets"]
        e.close()
    o = torch.zeros((n, n), dtype=torch.float64, device="cuda")
    s = torch.cuda.current_stream()
    check(lib().qk_finalize_fixed(ctypes.c_void_p(A.data_ptr()), n, ctypes.c_void_p(o.data_ptr()),
                                  ctypes.c_void_p(s.cuda_stream)), "qk_finalize_fixed")
    torch.cuda.synchronize()
    assert got_listed == listed            # the shards partition the work
    assert torch.equal(o, want)            # exact integer sums: bit for bit
    ref.close()


def test_one_shard_and_bad_arguments():
    _cuda()
    from quick_b200._native import QuickError
    from quick_b200.get2e import Get2e
    b = build_basis(water_cluster(2, 5.0, seed=1), "6-31G*")
    Dt = torch.eye(b.nbasis, dtype=torch.float64, device="cuda") * 0.5
    eng = Get2e(b, integral_cutoff=1e-10, prim_limit=1e-11)
    want = eng.fock2e(Dt)
    eng.set_shard(0, 1)
    assert torch.equal(eng.fock2e_sharded(Dt), want)   # no process group: one shard, no collective
    for rank, count in [(2, 2), (-1, 2), (0, 0)]:
        with pytest.raises(QuickError):
            eng.set_shard(rank, count)
    with pytest.raises(ValueError):
        eng.accumulate(Dt, torch.zeros((b.nbasis, b.nbasis), dtype=torch.float64, device="cuda"))
    eng.close()
