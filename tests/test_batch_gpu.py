"""GPU tests of the many-molecule Fock build (``qk_batch_fock2e``).

The batch merges the work lists of all molecules per integral class and runs one
launch per class, so every molecule sees exactly the quartets (and the int64
accumulation order does not matter) of its own one-molecule build: the results
must equal ``qk_fock2e_device`` bit for bit, and those are checked against the
oracle in the one-molecule tests."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from quick_b200.basis import build_basis  # noqa: E402
from quick_b200.molecules import water_cluster, alkane  # noqa: E402


def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _density(n, seed):
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(n, n)) * 0.15
    return torch.tensor(X @ X.T / n ** 0.5, device="cuda")


MOLS = [
    ("w1-sto3g", lambda: water_cluster(1, 6.0, seed=1), "STO-3G"),
    ("w3-631gs", lambda: water_cluster(3, 6.5, seed=2), "6-31G*"),
    ("c4h10-631gss", lambda: alkane(4), "6-31G**"),
    ("w5-sto3g", lambda: water_cluster(5, 7.0, seed=3), "STO-3G"),
    ("w1-ccpvtz", lambda: water_cluster(1, 6.0, seed=4), "CC-PVTZ"),
    ("w2-631gs", lambda: water_cluster(2, 6.0, seed=5), "6-31G*"),
]


@pytest.fixture(scope="module")
def engines():
    _cuda()
    from quick_b200.get2e import Get2e
    out = []
    for i, (name, molf, bas) in enumerate(MOLS):
        b = build_basis(molf(), bas)
        out.append((name, Get2e(b, integral_cutoff=1e-9, prim_limit=1e-10), _density(b.nbasis, 10 + i)))
    yield out
    for _, e, _ in out:
        e.close()


def test_batch_equals_single_bitwise(engines):
    from quick_b200.get2e import Get2eBatch
    singles = [e.fock2e(D).cpu().numpy() for _, e, D in engines]
    bt = Get2eBatch()
    got = bt.fock2e([e for _, e, _ in engines], [D for _, _, D in engines])
    for (name, _, _), s, g in zip(engines, singles, got):
        assert g.cpu().numpy().tobytes() == s.tobytes(), name
    # the cached merged lists are reused on the next call with the same molecules
    got2 = bt.fock2e([e for _, e, _ in engines], [D for _, _, D in engines])
    for (name, _, _), s, g in zip(engines, singles, got2):
        assert g.cpu().numpy().tobytes() == s.tobytes(), name
    bt.close()


def test_batch_subsets_and_order(engines):
    from quick_b200.get2e import Get2eBatch
    singles = {name: e.fock2e(D).cpu().numpy() for name, e, D in engines}
    bt = Get2eBatch()
    for pick in ([4, 0], [1, 2, 3], [5, 3, 1, 0], [2]):
        sel = [engines[i] for i in pick]
        got = bt.fock2e([e for _, e, _ in sel], [D for _, _, D in sel])
        for (name, _, _), g in zip(sel, got):
            assert g.cpu().numpy().tobytes() == singles[name].tobytes(), (pick, name)
    bt.close()


def test_batch_accumulates_into_o_and_takes_cutmat(engines):
    from quick_b200.get2e import Get2eBatch
    sel = engines[:3]
    os = [torch.full_like(D, 0.5) for _, _, D in sel]
    cms = [e.density_cutoff(D) for _, e, D in sel]
    ref = [e.fock2e(D, o=torch.full_like(D, 0.5), cutmat=c).cpu().numpy() for (_, e, D), c in zip(sel, cms)]
    bt = Get2eBatch()
    got = bt.fock2e([e for _, e, _ in sel], [D for _, _, D in sel], os=os, cutmats=cms)
    for (name, _, _), r, g, o in zip(sel, ref, got, os):
        assert g is o
        assert g.cpu().numpy().tobytes() == r.tobytes(), name
    bt.close()


def test_batch_mixed_precision_per_molecule(engines):
    from quick_b200.get2e import Get2eBatch
    _, e_mixed, D_mixed = engines[1]
    e_mixed.set_precision(1e-5)
    try:
        singles = [e.fock2e(D).cpu().numpy() for _, e, D in engines]
        assert e_mixed.fp32_quartets() > 0
        bt = Get2eBatch()
        got = bt.fock2e([e for _, e, _ in engines], [D for _, _, D in engines])
        for (name, _, _), s, g in zip(engines, singles, got):
            assert g.cpu().numpy().tobytes() == s.tobytes(), name
        bt.close()
    finally:
        e_mixed.set_precision(0.0)


def test_batch_rejects_duplicate_context(engines):
    from quick_b200.get2e import Get2eBatch
    from quick_b200._native import QuickError
    _, e, D = engines[0]
    bt = Get2eBatch()
    with pytest.raises(QuickError):
        bt.fock2e([e, e], [D, D])
    bt.close()


def test_batch_many_small_molecules():
    _cuda()
    from quick_b200.get2e import Get2e, Get2eBatch
    engs, Ds = [], []
    for i in range(24):
        b = build_basis(water_cluster(1 + i % 4, 6.0, seed=100 + i), "6-31G*" if i % 2 else "STO-3G")
        engs.append(Get2e(b, integral_cutoff=1e-9, prim_limit=1e-10))
        Ds.append(_density(b.nbasis, 200 + i))
    singles = [e.fock2e(D).cpu().numpy() for e, D in zip(engs, Ds)]
    bt = Get2eBatch()
    got = bt.fock2e(engs, Ds)
    for i, (s, g) in enumerate(zip(singles, got)):
        assert g.cpu().numpy().tobytes() == s.tobytes(), i
    bt.close()
    for e in engs:
        e.close()
