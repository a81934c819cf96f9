"""Host-side tests of the serving workload and its bookkeeping (no GPU)."""
import math

import numpy as np

from quick_b200.basis import A_TO_BOHRS, build_basis
from quick_b200.molecules import water_cluster
from quick_b200.serve import (TIP3P_H, TIP3P_O, Result, cluster_box, context_bytes_estimate, request_stream,
                              scf_bytes, summarize)


def test_stream_shape():
    reqs = request_stream(400, rate=50.0, seed=11)
    assert len(reqs) == 400
    arr = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(arr) > 0)
    # Poisson arrivals: mean gap 1/rate (400 samples: within 15 %)
    assert abs(np.mean(np.diff(arr)) - 1 / 50.0) < 0.15 / 50.0
    qm = [r for r in reqs if r.kind == "qmmm"]
    assert 0.18 < len(qm) / len(reqs) < 0.32
    for r in reqs:
        assert r.basis in ("STO-3G", "6-31G*")
        if r.kind == "molecule":
            nw = r.mol.natom // 3
            assert 1 <= nw <= 40 and r.mol.natom == 3 * nw
            assert r.ext_charges is None and r.series is None
        else:
            assert r.mol.natom == 60 and r.series is not None
            pos, q = r.ext_charges
            assert pos.shape == (4000, 3) and q.shape == (4000,)


def test_stream_sizes_log_uniform():
    reqs = [r for r in request_stream(1500, rate=100.0, seed=5, qmmm_fraction=0.0)]
    n = np.array([r.mol.natom // 3 for r in reqs])
    # log-uniform on [1, 40]: median near sqrt(40) ~ 6.3, a quarter below ~2.5
    assert 4 <= np.median(n) <= 9
    assert 0.15 < np.mean(n <= 2) < 0.35
    assert n.max() == 40 and n.min() == 1


def test_qmmm_series_random_walk_and_charges():
    reqs = [r for r in request_stream(300, rate=100.0, seed=3) if r.kind == "qmmm"]
    by = {}
    for r in reqs:
        by.setdefault(r.series, []).append(r)
    for s, rs in by.items():
        assert all(x.basis == rs[0].basis for x in rs)
        for a, b in zip(rs, rs[1:]):
            d = (b.mol.xyz - a.mol.xyz) / A_TO_BOHRS
            # one repeat moves each coordinate by N(0, 0.01 A)
            assert 0.003 < d.std() < 0.02
            assert np.array_equal(a.mol.Z, b.mol.Z)
        pos, q = rs[0].ext_charges
        assert np.allclose(q[0::3], TIP3P_O) and np.allclose(q[1::3], TIP3P_H)
        c = rs[0].mol.xyz.mean(axis=0)
        # O inside 15 A; an H can reach one O-H bond further
        assert np.max(np.linalg.norm(pos[0::3] - c, axis=1)) <= 15.0 * A_TO_BOHRS * 1.01
        assert np.max(np.linalg.norm(pos - c, axis=1)) <= 16.0 * A_TO_BOHRS
        dmin = np.min(np.linalg.norm(pos[:, None, :] - rs[0].mol.xyz[None], axis=2))
        assert dmin >= 1.9 * A_TO_BOHRS
        # rigid TIP3P waters (one random-walk step of 0.01 A away from 0.9572 A)
        oh = np.linalg.norm(pos[1::3][:1300] - pos[0::3][:1300], axis=1) / A_TO_BOHRS
        assert abs(np.median(oh) - 0.9572) < 0.02
        assert abs(q.sum() - TIP3P_O) < 1e-12          # 1333 neutral waters + one O charge


def test_stream_is_seeded():
    a = request_stream(50, rate=20.0, seed=9)
    b = request_stream(50, rate=20.0, seed=9)
    for x, y in zip(a, b):
        assert x.arrival == y.arrival and x.basis == y.basis
        assert np.array_equal(x.mol.xyz, y.mol.xyz)


def test_cluster_box_matches_named_workloads():
    assert cluster_box(1) == 6.0
    assert abs(cluster_box(32) - 10.0) < 0.1
    water_cluster(40, cluster_box(40), seed=1)   # placeable


def test_memory_estimates_grow():
    b1 = build_basis(water_cluster(2, 6.0, seed=1), "6-31G*")
    b2 = build_basis(water_cluster(8, cluster_box(8), seed=1), "6-31G*")
    assert 0 < context_bytes_estimate(b1) < context_bytes_estimate(b2)
    assert scf_bytes(100) == 8 * 100 * 100 * 34


def test_summarize_percentiles():
    rs = [Result(i, 0.0, 10, True, 7, "STO-3G", "molecule", 0.0, 0.0, (i + 1) / 1000.0, 0) for i in range(100)]
    s = summarize(rs, wall=2.0)
    assert s["requests"] == 100 and s["solves_per_s"] == 50.0
    assert math.isclose(s["p50_ms"], 50.5) and math.isclose(s["p99_ms"], 99.01)


def test_molecule_only_estimate_matches_basis():
    from quick_b200.serve import basis_size, request_bytes_estimate, request_bytes_estimate_mol
    for r in request_stream(20, rate=100.0, seed=12):
        b = build_basis(r.mol, r.basis)
        assert basis_size(r.mol, r.basis) == (b.nbasis, int(b.kprim.sum()))
        assert request_bytes_estimate_mol(r.mol, r.basis) == request_bytes_estimate(b)
