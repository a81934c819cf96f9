"""GPU tests of the launch-shape autotuner: every launch shape gives the same
Fock matrix bit for bit (persistent grids over the same work items), and the
tuner leaves the fastest measured shape applied."""
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from quick_b200.basis import build_basis  # noqa: E402
from quick_b200.molecules import water_cluster  # noqa: E402


def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _setup(nw=4, bas="6-31G*"):
    from quick_b200.get2e import Get2e
    b = build_basis(water_cluster(nw, 6.5, seed=11), bas)
    eng = Get2e(b, integral_cutoff=1e-10, prim_limit=1e-11)
    g = torch.Generator(device="cpu").manual_seed(3)
    X = torch.randn(b.nbasis, b.nbasis, generator=g, dtype=torch.float64) * 0.1
    D = (X @ X.T).cuda()
    return eng, D


def test_every_launch_shape_gives_the_same_fock_matrix():
    _cuda()
    from quick_b200 import autotune as at
    eng, D = _setup()
    ref = eng.fock2e(D).cpu().numpy()
    cls = at.classes(eng)
    for w in (1, 2, 3, 8):
        for i, _, mw in cls:
            at.set_shape(eng, i, min(w, mw), blocks_per_sm=(1 if w == 3 else 0))
        for s in (0, 1, 4):
            eng.set_streams(s)
            assert eng.fock2e(D).cpu().numpy().tobytes() == ref.tobytes(), (w, s)
    eng.close()


def test_tune_applies_the_fastest_shape():
    _cuda()
    from quick_b200 import autotune as at
    eng, D = _setup()
    ref = eng.fock2e(D).cpu().numpy()
    rep = at.tune(eng, D, warps=(2, 4), streams=(0, 4), reps=2)
    assert rep["best_streams"] in (0, 4)
    assert rep["ms_tuned"] == min(list(rep["streams"].values()) + list(rep["streams_merged_sp"].values()))
    assert rep["merge_sp"] in (False, True)
    for name, w in rep["warps"].items():
        assert w == min(rep["class_ms"][name], key=rep["class_ms"][name].get)
    assert eng.fock2e(D).cpu().numpy().tobytes() == ref.tobytes()
    eng.close()


def test_class_launch_rejects_bad_shapes():
    _cuda()
    from quick_b200 import autotune as at
    from quick_b200._native import QuickError
    eng, D = _setup(1, "STO-3G")
    with pytest.raises(QuickError):
        at.set_shape(eng, 0, 9)
    with pytest.raises(QuickError):
        at.set_shape(eng, 10 ** 6, 1)
    eng.close()


def test_tune_precision_stays_within_1_microhartree():
    _cuda()
    from quick_b200 import autotune as at
    from quick_b200.scf import RHF
    b = build_basis(water_cluster(3, 6.0, seed=2), "6-31G*")
    rep = at.tune_precision(lambda: RHF(b, integral_cutoff=1e-10), bounds=(1e-6, 1e-5), reps=2)
    assert rep["best_bound"] in (0.0, 1e-6, 1e-5)
    for bound, row in rep["bounds"].items():
        assert row["dE"] <= 1e-6, (bound, row)
