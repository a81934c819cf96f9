"""GPU test of the work lists built on the device (the default) against the host
builder (the reference implementation of the lists): per class the same quartet
and primitive-quartet counts and item counts, and the same Fock matrix bit for
bit, in plain FP64 and in the mixed form, for s/p/d and f shells."""
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


def _class_counts(eng):
    from quick_b200._native import lib
    L = lib()
    n = 64
    cls = np.zeros(4 * n, dtype=np.int32)
    ql = np.zeros(n, dtype=np.int64)
    pql = np.zeros(n, dtype=np.int64)
    P = lambda a: ctypes.c_void_p(a.ctypes.data)  # noqa: E731
    nc = L.qk_class_profile(ctypes.c_void_p(eng.h), n, P(cls), None, P(ql), P(pql), None, None, None, None)
    grids = []
    for ci in range(nc):
        g = ctypes.c_int(0)
        L.qk_class_launch(ctypes.c_void_p(eng.h), ci, None, None, None, ctypes.byref(g))
        grids.append(g.value)
    return ql[:nc].tolist(), pql[:nc].tolist(), grids


@pytest.mark.parametrize("bas,nw,bound", [("6-31G*", 6, 0.0), ("6-31G*", 6, 1e-5), ("CC-PVTZ", 2, 0.0),
                                          ("STO-3G", 10, 1e-6)])
def test_device_work_lists_equal_host_lists(bas, nw, bound):
    _cuda()
    from quick_b200.get2e import Get2e
    b = build_basis(water_cluster(nw, 7.0, seed=4), bas)
    rng = np.random.default_rng(8)
    X = rng.normal(size=(b.nbasis, b.nbasis)) * 0.15
    D = torch.tensor(X @ X.T / b.nbasis ** 0.5, device="cuda")
    out = {}
    for on_device in (0, 1):
        eng = Get2e(b, integral_cutoff=1e-10, prim_limit=1e-11)
        eng.set_worklist_builder(bool(on_device))
        eng.set_precision(bound)
        G = eng.fock2e(D).cpu().numpy()
        out[on_device] = (G, eng.work(), _class_counts(eng), eng.fp32_quartets())
        eng.close()
    (G0, w0, c0, f0), (G1, w1, c1, f1) = out[0], out[1]
    assert w0 == w1
    assert c0 == c1
    assert f0 == f1
    assert G0.tobytes() == G1.tobytes()
