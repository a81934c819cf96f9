"""World-size-2 tests of the multi-process logic on CPU (gloo): the job time is
the maximum over ranks, and a Fock build split over ranks by strided bra shells
(the reference's MPI split, src/mpi_setup.f90:295-354) sums back to the full
build after one all-reduce, and the int64 all-reduce that joins the shards of
a GPU build (Get2e.fock2e_sharded) is exact."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import sys
        root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
        sys.path.insert(0, root)
        import bench
        from oracle import oracle as O
        from quick_b200.basis import build_basis
        from quick_b200.molecules import water_cluster
        # 1. job time = the slowest rank's
        t = bench.max_over_ranks(10.0 + 5.0 * rank, dist, torch.device("cpu"))
        # 2. strided bra-shell shards, summed by one all-reduce
        b = build_basis(water_cluster(2, 5.0, seed=1), "STO-3G")
        orc = O.Oracle(b)
        Y, cp = orc.schwarz()
        D = np.eye(b.nbasis) * 0.6
        cm = orc.density_cutoff(D)
        G_part, _ = orc.get2e(D, cm, Y, cp, 1e-10, 1e-11, ii_range=(rank, 0), ii_stride=world)
        G = torch.tensor(G_part)
        dist.all_reduce(G)
        G_full, _ = orc.get2e(D, cm, Y, cp, 1e-10, 1e-11)
        # 3. the sharded GPU build's collective: int64 fixed-point accumulators summed
        #    exactly (quick_b200.get2e.allreduce_fixed, as Get2e.fock2e_sharded calls it)
        from quick_b200.get2e import allreduce_fixed
        parts = [np.random.default_rng(r).integers(-2 ** 52, 2 ** 52, size=(7, 7)) for r in range(world)]
        A = torch.tensor(parts[rank], dtype=torch.int64)
        allreduce_fixed(A)
        exact = bool((A.numpy() == parts[0] + parts[1]).all())
        q.put((rank, t, float(np.abs(G.numpy() - G_full).max()), exact))
    finally:
        dist.destroy_process_group()


def test_two_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, err, exact in out:
        assert t == 15.0
        assert err <= 1e-13
        assert exact
