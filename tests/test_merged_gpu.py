"""GPU test of the merged s/p launch (qk_set_merge_sp): the six per-lane s/p
classes as one persistent kernel per precision give the same Fock matrix bit for
bit as one launch per class, in plain FP64 and in the mixed form, with fewer
launches per build."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from quick_b200.basis import build_basis  # noqa: E402
from quick_b200.molecules import water_cluster  # noqa: E402


@pytest.mark.parametrize("bas,nw,bound", [("STO-3G", 10, 0.0), ("6-31G*", 4, 0.0), ("6-31G*", 4, 1e-5),
                                          ("CC-PVTZ", 1, 0.0)])
def test_merged_sp_launch_equals_per_class_launches(bas, nw, bound):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from quick_b200.get2e import Get2e
    b = build_basis(water_cluster(nw, 7.0, seed=6), bas)
    rng = np.random.default_rng(11)
    X = rng.normal(size=(b.nbasis, b.nbasis)) * 0.15
    D = torch.tensor(X @ X.T / b.nbasis ** 0.5, device="cuda")
    out = {}
    for merged in (False, True):
        eng = Get2e(b, integral_cutoff=1e-10, prim_limit=1e-11)
        eng.set_precision(bound)
        eng.set_merge_sp(merged)
        Gs = [eng.fock2e(D).cpu().numpy() for _ in range(2)]
        out[merged] = (Gs, eng.work()["launches"])
        eng.close()
    (G0, l0), (G1, l1) = out[False], out[True]
    assert G0[0].tobytes() == G0[1].tobytes() == G1[0].tobytes() == G1[1].tobytes()
    assert l1 < l0, (l0, l1)


def test_allocation_free_build_reports_its_own_launches():
    """With the merged option set, the allocation-free build still launches one
    kernel per class; qk_last_work reports the launches of the build that ran."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import ctypes
    from quick_b200._native import check, lib
    from quick_b200.get2e import Get2e
    b = build_basis(water_cluster(3, 6.0, seed=6), "STO-3G")
    rng = np.random.default_rng(12)
    X = rng.normal(size=(b.nbasis, b.nbasis)) * 0.15
    D = torch.tensor(X @ X.T / b.nbasis ** 0.5, device="cuda")
    eng = Get2e(b, integral_cutoff=1e-10, prim_limit=1e-11)
    eng.set_merge_sp(True)
    G_merged = eng.fock2e(D).cpu().numpy()
    merged = eng.work()["launches"]
    o = torch.zeros_like(D)
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    check(lib().qk_fock2e_device_noalloc(ctypes.c_void_p(eng.h), ctypes.c_void_p(D.data_ptr()), None,
                                         ctypes.c_void_p(o.data_ptr()), s), "qk_fock2e_device_noalloc")
    torch.cuda.synchronize()
    per_class = eng.work()["launches"]
    eng.close()
    assert per_class > merged
    assert np.abs(o.cpu().numpy() - G_merged).max() == 0.0
