"""SCF request serving on one GPU around the batched Fock build.

A request is one closed-shell RHF solve: a molecule and a basis, optionally with
external point charges (a QM/MM step) and a series it belongs to.  The server
keeps every admitted solve resident on the device -- its :class:`Get2e` context
(shell-pair tables, work lists, Schwarz bounds), its density, Fock matrices and
DIIS history -- and advances all of them together: each step is ONE batched
Fock build over every active molecule (``qk_batch_fock2e``: per integral class
one launch over the merged work lists of all molecules), followed by each
solve's DIIS / density update on the device and one host synchronisation for
the convergence test of all solves.  Solves join and leave between steps
(continuous batching); a QM/MM repeat starts from the last converged density of
its series, which stays on the device.

Admission is by a device-memory budget: a request is admitted (first come,
first served) when the bytes it will hold -- its context (estimated, then
measured once built) plus its SCF matrices -- fit beside the solves already
running.  Latency of a request = completion time - arrival
time; the server reports p50 / p99 beside throughput.

The per-solve arithmetic is :class:`quick_b200.scf.DeviceSCFState` -- that of
the graph-captured SCF (``GraphSCF``) -- or :class:`quick_b200.scf.SCFState`, the
eager loop of ``RHF.run``; a batched Fock build equals the one-molecule build
bit for bit, so a request's result does not depend on what else was in the
batch.

The reference (QUICK) computes one molecule per process and has no server; the
QM/MM step it serves is the Fortran API's ``get_quick_energy`` call with new
coordinates and point charges (``src/modules/quick_api_module.f90:373-404``),
with the previous density reused when ``reusedmx`` is set
(``quick_api_module.f90:183-291``) -- what a QM/MM repeat stands for here.
"""
from __future__ import annotations

import math
import threading
import time
from collections import deque
from concurrent.futures import FIRST_COMPLETED, ThreadPoolExecutor, wait
from dataclasses import dataclass, field

import numpy as np

from ._native import free_stream, own_stream
from .basis import A_TO_BOHRS, Molecule, build_basis
from .molecules import water_cluster

# TIP3P point charges (e)
TIP3P_O, TIP3P_H = -0.834, 0.417


@dataclass
class Request:
    rid: int
    mol: Molecule
    basis: str
    arrival: float = 0.0                 # seconds after the start of the stream
    ext_charges: tuple = None            # (positions (n, 3) Bohr, charges (n,))
    series: int = None                   # QM/MM series: warm start from its last density
    kind: str = "molecule"


@dataclass
class Result:
    rid: int
    E: float
    niter: int
    converged: bool
    nbasis: int
    basis: str
    kind: str
    arrival: float
    admitted: float
    done: float
    bytes: int
    warm: bool = False
    D: object = field(default=None, repr=False)

    @property
    def latency(self):
        return self.done - self.arrival


def cluster_box(n: int) -> float:
    """Cube edge (Angstrom) for an n-water cluster: about the density of the
    named cluster workloads (4 waters in 6 A, 12 in 8 A, 32 in 10 A)."""
    return max(6.0, 3.15 * n ** (1.0 / 3.0))


def _point_charges(rng, qm_xyz_bohr, n, radius_ang, exclude_ang=2.0):
    """n TIP3P point charges around the QM centroid: n // 3 rigid TIP3P waters
    (O -0.834 e, two H +0.417 e; O-H 0.9572 A, H-O-H 104.52 deg) with their O
    uniform in a sphere of ``radius_ang`` and random orientations, plus n % 3 lone
    O charges; every charge at least ``exclude_ang`` from every QM atom.  MM
    waters may overlap one another (they are only charges)."""
    from .molecules import _rand_rotation
    c = qm_xyz_bohr.mean(axis=0)
    R = radius_ang * A_TO_BOHRS
    ex2 = (exclude_ang * A_TO_BOHRS) ** 2
    r, ang = 0.9572 * A_TO_BOHRS, math.radians(104.52)
    local = np.array([[0.0, 0.0, 0.0],
                      [r * math.sin(ang / 2), 0.0, r * math.cos(ang / 2)],
                      [-r * math.sin(ang / 2), 0.0, r * math.cos(ang / 2)]])
    nw, nlone = n // 3, n % 3
    pos, q = [], []

    def far(x):
        return ((x[:, None, :] - qm_xyz_bohr[None, :, :]) ** 2).sum(-1).min() >= ex2

    while len(pos) < 3 * nw:
        o = rng.uniform(-R, R, size=3)
        if o @ o > R * R:
            continue
        w = c + o + local @ _rand_rotation(rng).T
        if far(w):
            pos.extend(w)
            q.extend([TIP3P_O, TIP3P_H, TIP3P_H])
    while len(pos) < n:
        o = rng.uniform(-R, R, size=3)
        if o @ o <= R * R and far((c + o)[None, :]):
            pos.append(c + o)
            q.append(TIP3P_O)
    return np.array(pos), np.array(q)


def _independent_charges(rng, qm_xyz_bohr, n, radius_ang, exclude_ang=2.0):
    """n independent point charges, each uniform in a sphere of ``radius_ang``
    around the QM centroid and at least ``exclude_ang`` from every QM atom: a third
    with the TIP3P oxygen charge (-0.834 e), the rest with the hydrogen charge
    (+0.417 e), so the set is about neutral but has no local (molecular) neutrality."""
    c = qm_xyz_bohr.mean(axis=0)
    R = radius_ang * A_TO_BOHRS
    ex2 = (exclude_ang * A_TO_BOHRS) ** 2
    pos = []
    while len(pos) < n:
        o = rng.uniform(-R, R, size=3)
        x = c + o
        if o @ o <= R * R and ((qm_xyz_bohr - x) ** 2).sum(-1).min() >= ex2:
            pos.append(x)
    q = np.full(n, TIP3P_H)
    q[: n // 3] = TIP3P_O
    return np.array(pos), q


def request_stream(n_requests: int, rate: float, seed: int = 20261203, qmmm_fraction: float = 0.25,
                   max_waters: int = 40, bases=("STO-3G", "6-31G*"), qm_waters: int = 20,
                   n_charges: int = 4000, charge_radius: float = 15.0, sigma: float = 0.01,
                   n_series: int = 16, charges: str = "waters"):
    """The serving workload: ``n_requests`` RHF requests with Poisson arrivals at
    ``rate`` per second.

    * molecules: seeded water clusters with N log-uniform in [1, max_waters]
      (box from :func:`cluster_box`), basis uniform over ``bases``;
    * a ``qmmm_fraction`` of requests are QM/MM repeats: ``n_series`` series,
      each a ``qm_waters`` QM region with ``n_charges`` TIP3P point charges (MM
      waters, :func:`_point_charges`) within ``charge_radius`` A; every repeat
      moves the QM atoms and the charges of its series by Gaussian ``sigma`` A (a
      random walk), and is solved from the series' last density.  ``charges``:
      "waters" (the default) places the charges as rigid TIP3P waters;
      "independent" places each charge on its own (:func:`_independent_charges`).
    """
    if charges not in ("waters", "independent"):
        raise ValueError("charges: 'waters' or 'independent'")
    place = _point_charges if charges == "waters" else _independent_charges
    rng = np.random.Generator(np.random.PCG64(seed))
    series = []
    for s in range(n_series):
        mol = water_cluster(qm_waters, cluster_box(qm_waters), seed=seed + 7919 * (s + 1))
        pos, q = place(rng, mol.xyz, n_charges, charge_radius)
        series.append({"mol": mol, "pos": pos, "q": q, "basis": bases[s % len(bases)]})
    out = []
    t = 0.0
    lo, hi = 0.0, math.log(max_waters)
    for i in range(n_requests):
        t += rng.exponential(1.0 / rate)
        if rng.random() < qmmm_fraction:
            s = int(rng.integers(n_series))
            S = series[s]
            sb = sigma * A_TO_BOHRS
            S["mol"] = Molecule(Z=S["mol"].Z, xyz=S["mol"].xyz + rng.normal(scale=sb, size=S["mol"].xyz.shape))
            S["pos"] = S["pos"] + rng.normal(scale=sb, size=S["pos"].shape)
            out.append(Request(i, S["mol"], S["basis"], t, (S["pos"], S["q"]), s, "qmmm"))
        else:
            n = int(min(max_waters, max(1, round(math.exp(rng.uniform(lo, hi))))))
            mol = water_cluster(n, cluster_box(n), seed=int(rng.integers(1 << 31)))
            out.append(Request(i, mol, bases[int(rng.integers(len(bases)))], t))
    return out


def scf_bytes(nbasis: int, maxdiis: int = 10) -> int:
    """Device bytes of one solve's SCF matrices: S, H, X, D, D_prev, the new D,
    F, F_prev, 2 * maxdiis DIIS vectors and about 6 temporaries of the step."""
    return 8 * nbasis * nbasis * (2 * maxdiis + 14)


def context_bytes_estimate(basis) -> int:
    """Estimate of a context's device bytes before its tables are built: 1 MiB
    of fixed buffers, 88 bytes per primitive pair, and 400 bytes per nbasis^2
    for the int64 accumulator, the density screen and the work lists (measured
    on the water clusters of the serving stream: 130 B/nbasis^2 and less for
    40 waters).  Replaced by the measured figure after the request's first
    Fock build."""
    prims = int(np.asarray(basis.kprim, dtype=np.int64).sum())
    n = basis.nbasis
    return (1 << 20) + 88 * prims * prims + 400 * n * n


def request_bytes_estimate(basis, maxdiis: int = 10) -> int:
    """Bytes a request is admitted against before its tables exist."""
    return context_bytes_estimate(basis) + scf_bytes(basis.nbasis, maxdiis)


_ELEMENT_SIZES = {}


def basis_size(mol, name: str):
    """(nbasis, primitives summed over shells) of ``mol`` in basis ``name``, from
    per-element counts (no basis arrays built)."""
    from .basis import SYMBOLS, load_basis_data
    nfun = {"S": 1, "P": 3, "SP": 4, "D": 6, "F": 10}
    nb = npr = 0
    for z in mol.Z:
        key = (name, int(z))
        if key not in _ELEMENT_SIZES:
            data = load_basis_data(name)[SYMBOLS[int(z)]]
            _ELEMENT_SIZES[key] = (sum(nfun[k] for k, _ in data), sum(len(p) for _, p in data))
        a, b = _ELEMENT_SIZES[key]
        nb += a
        npr += b
    return nb, npr


def request_bytes_estimate_mol(mol, name: str, maxdiis: int = 10) -> int:
    """:func:`request_bytes_estimate` from the molecule and basis name."""
    n, prims = basis_size(mol, name)
    return (1 << 20) + 88 * prims * prims + 400 * n * n + scf_bytes(n, maxdiis)


class _Job:
    __slots__ = ("req", "eng", "rhf", "st", "bytes", "measured", "admitted", "warm", "lane", "load", "cohort")


class Server:
    """Continuous-batching SCF server on one GPU (see the module docstring).

    ``memory_budget``: device bytes that the admitted solves (and the contexts
    kept for reuse) may hold; default half of the free device memory at start.
    ``fp32_bound``: the mixed form's Schwarz bound product below which quartets
    run in FP32 (0 = plain FP64).  ``max_active``: cap on solves in one batch.
    ``pool``: retired contexts kept for the next requests (their device buffers
    are reused by ``Get2e.bind``; allocation and release synchronise the GPU).
    ``workers``: threads that set new requests up (basis, context, pair tables,
    one-electron integrals, guess) on their own CUDA streams while the batch
    steps go on; 0 sets them up inline, so that every request admitted at a step
    is in that step's batch.
    ``scf``: "device" advances each solve with :class:`DeviceSCFState` (DIIS on
    the device, SP2 density: no host synchronisation inside a step; the
    post-build half of its cycle captured once as a CUDA graph); "eigh" with
    :class:`SCFState` (torch eigh, one synchronisation per solve and step).
    ``lanes``: streams (each with its own graph memory pool) over which the
    solves' post-build graphs are spread; a solve keeps its lane, and joins the
    one with the least SP2 work (sum of m^3) at admission.  The post-build half is
    a chain of small kernels per solve, so solves on different lanes overlap.
    ``post_graph``: capture each solve's post-build half as a CUDA graph (else it
    runs eagerly on its lane).
    ``pipeline``: split the solves into two cohorts stepped in turn, so that one
    cohort's post-build halves and read-back run while the other's Fock build
    runs, and the host takes one cohort's figures while the GPU works on the other;
    ``reserve_sms`` then leaves that many SMs to the post-build kernels while a
    batch's persistent Fock kernels run."""

    def __init__(self, device: int = 0, memory_budget: int = None, fp32_bound: float = 0.0,
                 denserms: float = 1e-6, maxiter: int = 100, integral_cutoff: float = 1e-10,
                 max_active: int = 512, maxdiis: int = 10, keep_densities: bool = False, pool: int = 64,
                 workers: int = 4, scf: str = "device", reserve_sms: int = 0, lanes: int = 4,
                 post_graph: bool = True, pipeline: bool = True):
        import torch
        from .get2e import Get2eBatch
        self.torch = torch
        self.device = device
        torch.cuda.set_device(device)
        if memory_budget is None:
            free, _ = torch.cuda.mem_get_info(device)
            memory_budget = free // 2
        self.budget = int(memory_budget)
        self.fp32_bound = float(fp32_bound)
        self.denserms, self.maxiter, self.maxdiis = denserms, maxiter, maxdiis
        self.integral_cutoff = integral_cutoff
        self.max_active = max_active
        self.keep_densities = keep_densities
        self.pool_max = pool
        self.pool = []                # (Get2e, bytes) kept for reuse
        self._arrival = lambda r: r.arrival
        self.batch = Get2eBatch(device)
        # reserve_sms > 0 leaves SMs to the set-up threads' kernels while a batch's
        # persistent kernels run (measured: no gain beyond the run-to-run spread)
        self.batch.reserve_sms(reserve_sms)
        self.active = []
        self.queue = deque()
        self.series_D = {}            # series -> last converged density (device)
        self.series_busy = set()      # series with a request in flight
        self.used = 0
        self.peak_used = 0
        self.steps = 0
        self.batch_sizes = []
        self.max_concurrent = 0       # most solves in flight at once
        self.rejected = []
        self.timers = {"admit": 0.0, "setup_engine": 0.0, "setup_rhf": 0.0, "fock": 0.0, "scf": 0.0, "sync": 0.0,
                       "retire": 0.0, "fock_gpu": 0.0}
        self._ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        # set-up of new requests runs on its own streams, beside the batch's builds
        self.main_stream = torch.cuda.current_stream(device)
        self.workers = workers
        self.scf = scf
        # torch initialises its linear-algebra back end lazily and not thread-safely:
        # do it here, before the set-up threads call eigh / solve for the first time
        a = torch.eye(4, dtype=torch.float64, device=torch.device("cuda", device)) * 2.0
        torch.linalg.eigh(a)
        torch.linalg.solve_ex(a, a[0])
        (a @ a).sum().item()
        self.executor = ThreadPoolExecutor(max_workers=workers) if workers > 0 else None
        self._tls = threading.local()
        self._own_streams = []        # streams this server took (set-up threads, read-back), given back by close()
        self.lanes = max(1, int(lanes))
        self.post_graph = post_graph
        # two cohorts stepped in turn (device SCF only): one's post-build halves and
        # read-back run while the other's Fock build runs.  Each has its own batch
        # (a batch's staging block serves one build in flight), read-back stream and
        # pinned buffer of convergence figures.
        self.pipeline = bool(pipeline) and scf == "device"
        self.cohorts = [[], []]
        self.cohort_load = [0.0, 0.0]
        self._inflight = [None, None]
        if self.pipeline:
            self.batches = [self.batch, Get2eBatch(device)]
            self.batches[1].reserve_sms(reserve_sms)
            self._rb = [own_stream(device), own_stream(device)]
            self._own_streams.extend(self._rb)
            self._pinned = [torch.zeros((max_active, 4), dtype=torch.float64).pin_memory() for _ in range(2)]
            self._step_done = [None, None]
        self.lane_load = [0.0] * self.lanes
        self._streams_lock = threading.Lock()
        self.setting_up = []          # (future, request, reserved bytes, admission time)

    # -- admission
    def _stream(self):
        st = getattr(self._tls, "stream", None)
        if st is None:
            self.torch.cuda.set_device(self.device)
            # high priority: the set-up's kernels get SMs at the batch kernels' boundaries;
            # a stream of its own, never one that a graph capture may be using
            st = self._tls.stream = own_stream(self.device)
            with self._streams_lock:
                self._own_streams.append(st)
        return st

    def _setup(self, req, eng, D0):
        """Set one request up (worker thread or inline): returns the context, the
        RHF object, the SCF state and an event marking the end of its GPU work."""
        from .get2e import Get2e
        from .scf import RHF, DeviceSCFState
        torch = self.torch
        stream = self._stream()
        t = time.perf_counter()
        basis = build_basis(req.mol, req.basis)
        if eng is None:
            eng = Get2e(basis, device=self.device, integral_cutoff=self.integral_cutoff,
                        prim_limit=0.1 * self.integral_cutoff)
            if self.fp32_bound > 0.0:
                eng.set_precision(self.fp32_bound)
        else:
            eng.bind(basis)
        eng.prepare()
        t1 = time.perf_counter()
        D0, D0_ready = D0 if isinstance(D0, tuple) else (D0, None)
        with torch.cuda.stream(stream):
            if D0_ready is not None:
                stream.wait_event(D0_ready)
            rhf = RHF(basis, device=self.device, ext_charges=req.ext_charges, engine=eng)
            if self.scf == "device":
                st = DeviceSCFState(rhf, denserms=self.denserms, maxiter=self.maxiter, D0=D0, maxdiis=self.maxdiis,
                                    graph=self.post_graph)
            else:
                st = rhf.state(denserms=self.denserms, maxiter=self.maxiter, maxdiis=self.maxdiis, D0=D0)
            ev = torch.cuda.Event()
            ev.record(stream)
        self.timers["setup_engine"] += t1 - t
        self.timers["setup_rhf"] += time.perf_counter() - t1
        return eng, rhf, st, ev

    def _join(self, req, est, admitted, result):
        eng, rhf, st, ev = result
        self.main_stream.wait_event(ev)
        j = _Job()
        j.req, j.eng, j.rhf, j.st = req, eng, rhf, st
        j.load = float(rhf.X.shape[1]) ** 3
        j.lane = min(range(self.lanes), key=lambda k: self.lane_load[k])
        self.lane_load[j.lane] += j.load
        if hasattr(st, "lane"):
            st.lane = j.lane
        if self.pipeline:
            j.cohort = 0 if self.cohort_load[0] <= self.cohort_load[1] else 1
            self.cohort_load[j.cohort] += j.load
            self.cohorts[j.cohort].append(j)
        j.warm = st.warm
        j.admitted = admitted
        j.measured = False
        j.bytes = est
        self.active.append(j)

    def _admit(self, now):
        """First come, first served among the admissible requests: a QM/MM repeat
        waits (without holding up the others) while its series has a request in
        flight, so that it starts from that request's density.  Memory is reserved
        here, before the set-up allocates anything."""
        t = time.perf_counter()
        skipped = deque()
        while self.queue and len(self.active) + len(self.setting_up) < self.max_active:
            req = self.queue[0]
            if req.series is not None and req.series in self.series_busy:
                skipped.append(self.queue.popleft())
                continue
            est = request_bytes_estimate_mol(req.mol, req.basis, self.maxdiis)
            if est > self.budget:
                self.queue.popleft()
                self.rejected.append((req.rid, est))
                continue
            while self.used + est > self.budget and self.pool:
                eng, b = self.pool.pop(0)
                self.used -= b
                eng.close()
            if self.used + est > self.budget and (self.active or self.setting_up):
                break                      # wait for memory
            self.queue.popleft()
            eng = None
            if self.pool:
                # the largest kept context: its buffers most likely fit without a
                # reallocation (cudaMalloc/cudaFree synchronise the whole GPU)
                i = max(range(len(self.pool)), key=lambda x: self.pool[x][1])
                eng, b = self.pool.pop(i)
                self.used -= b
            self.used += est
            self.peak_used = max(self.peak_used, self.used)
            D0 = self.series_D.get(req.series) if req.series is not None else None
            if req.series is not None:
                self.series_busy.add(req.series)
            if self.executor is None:
                self._join(req, est, now, self._setup(req, eng, D0))
            else:
                self.setting_up.append((self.executor.submit(self._setup, req, eng, D0), req, est, now))
        while skipped:
            self.queue.appendleft(skipped.pop())
        self.timers["admit"] += time.perf_counter() - t

    def _collect(self, block_until: float = None):
        """Requests whose set-up finished join the batch (optionally waiting up to
        ``block_until`` seconds for the first one)."""
        if not self.setting_up:
            return
        if block_until is not None:
            wait([f for f, _, _, _ in self.setting_up], timeout=max(0.0, block_until), return_when=FIRST_COMPLETED)
        keep = []
        for f, req, est, adm in self.setting_up:
            if f.done():
                self._join(req, est, adm, f.result())
            else:
                keep.append((f, req, est, adm))
        self.setting_up = keep

    # -- one step of every active solve, in two halves: the batched Fock build is
    # enqueued first, new requests are set up on the host and the side stream
    # while the GPU computes it, then every solve's DIIS / density update runs
    # and one host synchronisation reads all convergence figures.
    def _launch(self):
        act = self.active
        t0 = time.perf_counter()
        ins = [j.st.fock_input() for j in act]
        self._ev[0].record()
        self.batch.fock2e([j.eng for j in act], [d for d, _ in ins], os=[f for _, f in ins])
        self._ev[1].record()
        self.timers["fock"] += time.perf_counter() - t0
        return list(act)

    def _finish(self, act, clock):
        from .scf import DeviceSCFState
        torch = self.torch
        t1 = time.perf_counter()
        if self.scf == "device":
            v = DeviceSCFState.step_many([j.st for j in act])
        else:
            v = torch.stack([j.st.step_device() for j in act])
        t2 = time.perf_counter()
        vals = v.cpu().numpy()
        t3 = time.perf_counter()
        self.timers["scf"] += t2 - t1
        self.timers["sync"] += t3 - t2
        self.timers["fock_gpu"] += self._ev[0].elapsed_time(self._ev[1]) * 1e-3
        return self._absorb(act, vals, clock, self.main_stream)

    def _absorb(self, act, vals, clock, stream):
        """Every solve of a finished step takes its convergence figures; the
        converged ones retire (their density copies are made on ``stream``, on
        which the step's work is already complete or ordered)."""
        torch = self.torch
        t3 = time.perf_counter()
        self.steps += 1
        self.batch_sizes.append(len(act))
        self.max_concurrent = max(self.max_concurrent, len(self.active))
        done = []
        for j, v in zip(act, vals):
            if not j.measured:
                tot, _ = j.eng.device_bytes()
                b = tot + scf_bytes(j.rhf.basis.nbasis, self.maxdiis)
                self.used += b - j.bytes
                j.bytes = b
                j.measured = True
            j.st.step(v)
            if j.st.done:
                done.append(j)
        self.peak_used = max(self.peak_used, self.used)
        gone = {id(j) for j in done}
        self.active = [j for j in self.active if id(j) not in gone]
        if self.pipeline and gone:
            self.cohorts = [[j for j in c if id(j) not in gone] for c in self.cohorts]
        out = []
        if done:
            t = clock()
            with torch.cuda.stream(stream):
                rs = [j.st.result() for j in done]
                ev = torch.cuda.Event()
                ev.record(stream)
            # the copies read the solves' own buffers, which are freed (and may be
            # handed to a set-up thread's stream) as soon as the solves are dropped
            ev.synchronize()
            for j, r in zip(done, rs):
                self.lane_load[j.lane] -= j.load
                if self.pipeline:
                    self.cohort_load[j.cohort] -= j.load
                req = j.req
                if req.series is not None:
                    self.series_busy.discard(req.series)
                    if r["converged"]:
                        # the next request of the series starts from this density once
                        # its copy (ordered by ev) is done
                        self.series_D[req.series] = (r["D"], ev)
                out.append(Result(req.rid, r["E"], r["niter"], r["converged"], j.rhf.basis.nbasis, req.basis,
                                  req.kind, self._arrival(req), j.admitted, t, j.bytes, j.warm,
                                  r["D"] if self.keep_densities else None))
                self.used -= j.bytes
                if len(self.pool) < self.pool_max:
                    tot, _ = j.eng.device_bytes()
                    self.pool.append((j.eng, tot))
                    self.used += tot
                else:
                    j.eng.close()
        self.timers["retire"] += time.perf_counter() - t3
        return out

    # -- the pipelined step (two cohorts)
    def _launch_cohort(self, k):
        """Enqueue one step of cohort k: its batched Fock build on the main stream
        (ordered after the cohort's previous post-build halves), the post-build
        halves on the lanes, and the read-back of the convergence figures into
        pinned memory on the cohort's read-back stream."""
        from .scf import DeviceSCFState
        torch = self.torch
        act = list(self.cohorts[k])
        t0 = time.perf_counter()
        main = self.main_stream
        if self._step_done[k] is not None:
            main.wait_event(self._step_done[k])
        ins = [j.st.fock_input() for j in act]
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(main)
        self.batches[k].fock2e([j.eng for j in act], [d for d, _ in ins], os=[f for _, f in ins], stream=main)
        e1.record(main)
        t1 = time.perf_counter()
        rb = self._rb[k]
        v = DeviceSCFState.step_many([j.st for j in act], join=rb)
        host = self._pinned[k][: len(act)]
        with torch.cuda.stream(rb):
            host.copy_(v, non_blocking=True)
            done = torch.cuda.Event()
            done.record(rb)
        self._step_done[k] = done
        self.timers["fock"] += t1 - t0
        self.timers["scf"] += time.perf_counter() - t1
        return act, done, host, v, e0, e1

    def _finish_cohort(self, k, clock):
        act, done, host, v, e0, e1 = self._inflight[k]
        self._inflight[k] = None
        t = time.perf_counter()
        done.synchronize()
        vals = host.numpy().copy()
        self.timers["sync"] += time.perf_counter() - t
        self.timers["fock_gpu"] += e0.elapsed_time(e1) * 1e-3
        return self._absorb(act, vals, clock, self._rb[k])

    def serve(self, requests, realtime: bool = True):
        """Run a request stream to completion; returns the results in request order.

        ``realtime``: requests arrive at their ``arrival`` times (the loop sleeps
        while nothing is active); otherwise all are queued at the start and
        latencies count from the start."""
        arrival = (lambda r: r.arrival) if realtime else (lambda r: 0.0)
        pending = deque(sorted(requests, key=lambda r: (arrival(r), r.rid)))
        t0 = time.perf_counter()
        clock = lambda: time.perf_counter() - t0  # noqa: E731
        self._arrival = arrival
        results = []
        if self.pipeline:
            k = 0
            while pending or self.queue or self.active or self.setting_up or any(self._inflight):
                now = clock()
                while pending and arrival(pending[0]) <= now:
                    self.queue.append(pending.popleft())
                # cohort k: take its last step's figures (its post-build ran beside the
                # other cohort's Fock build), then launch its next step
                if self._inflight[k] is not None:
                    results.extend(self._finish_cohort(k, clock))
                self._admit(now)
                self._collect()
                if self.cohorts[k]:
                    self._inflight[k] = self._launch_cohort(k)
                if not any(self._inflight) and not self.active:
                    nxt = (arrival(pending[0]) - clock()) if pending else None
                    if self.setting_up:
                        self._collect(block_until=nxt if nxt is not None else 60.0)
                    elif nxt is not None and not self.queue:
                        time.sleep(max(0.0, nxt))
                k ^= 1
            self.wall = clock()
            return sorted(results, key=lambda r: r.rid)
        while pending or self.queue or self.active or self.setting_up:
            now = clock()
            while pending and arrival(pending[0]) <= now:
                self.queue.append(pending.popleft())
            act = self._launch() if self.active else None
            self._admit(now)
            if act:
                results.extend(self._finish(act, clock))
            if not self.active:
                nxt = (arrival(pending[0]) - clock()) if pending else None
                if self.setting_up:
                    self._collect(block_until=nxt if nxt is not None else 60.0)
                elif nxt is not None and not self.queue:
                    time.sleep(max(0.0, nxt))
            else:
                self._collect()
        self.wall = clock()
        return sorted(results, key=lambda r: r.rid)

    def close(self):
        self.torch.cuda.synchronize(self.device)
        if self.executor is not None:
            self.executor.shutdown(wait=True)
            for f, _, _, _ in self.setting_up:
                if f.done() and f.exception() is None:
                    f.result()[0].close()
            self.setting_up = []
        for j in self.active:
            j.eng.close()
        for eng, _ in self.pool:
            eng.close()
        self.active = []
        self.pool = []
        self.used = 0
        self.cohorts = [[], []]
        self._inflight = [None, None]
        self.batch.close()
        if self.pipeline:
            self.batches[1].close()
        if self._own_streams:
            self.torch.cuda.synchronize(self.device)
            for st in self._own_streams:
                free_stream(st)
            self._own_streams = []


def summarize(results, wall: float) -> dict:
    """Throughput and latency percentiles of a served stream."""
    lat = np.array([r.latency for r in results]) * 1e3
    return {
        "requests": len(results),
        "solves_per_s": len(results) / wall if wall > 0 else None,
        "wall_s": wall,
        "p50_ms": float(np.percentile(lat, 50)) if len(lat) else None,
        "p99_ms": float(np.percentile(lat, 99)) if len(lat) else None,
        "mean_iterations": float(np.mean([r.niter for r in results])) if results else None,
        "converged": int(sum(r.converged for r in results)),
    }


def run_sequential(requests, fp32_bound: float = 0.0, device: int = 0, denserms: float = 1e-6,
                   integral_cutoff: float = 1e-10, maxiter: int = 100, graph: bool = False):
    """The plain path the server is measured against: the same requests solved one
    at a time, in request order, with no batching -- per request its basis, its
    context (one context rebound to each molecule, as a caller of the one-molecule
    API would keep it), one-electron integrals with its point charges, the SAD
    guess (or its series' last density) and the device SCF cycle (``GraphSCF``),
    run eagerly (the default: one request at a time it is the faster form, the
    capture of two graphs per request costing more than their replays save) or
    captured as CUDA graphs (``graph=True``).
    Returns (summary, results); ``solves_per_s`` is the requests over the time
    to solve all of them back to back, arrivals ignored (the capacity of the
    plain path)."""
    import torch
    from .get2e import Get2e
    from .scf import RHF, GraphSCF
    torch.cuda.set_device(device)
    eng = None
    series_D = {}
    results = []
    t0 = time.perf_counter()
    for req in requests:
        ta = time.perf_counter() - t0
        basis = build_basis(req.mol, req.basis)
        if eng is None:
            eng = Get2e(basis, device=device, integral_cutoff=integral_cutoff, prim_limit=0.1 * integral_cutoff)
            if fp32_bound > 0.0:
                eng.set_precision(fp32_bound)
        else:
            eng.bind(basis)
        rhf = RHF(basis, device=device, ext_charges=req.ext_charges, engine=eng)
        D0 = series_D.get(req.series) if req.series is not None else None
        r = GraphSCF(rhf).run(denserms=denserms, maxiter=maxiter, D0=D0, graph=graph)
        if req.series is not None and r["converged"]:
            series_D[req.series] = r["D"]
        done = time.perf_counter() - t0
        results.append(Result(req.rid, r["E"], r["niter"], r["converged"], basis.nbasis, req.basis, req.kind,
                              ta, ta, done, 0, D0 is not None))
    wall = time.perf_counter() - t0
    if eng is not None:
        eng.close()
    s = summarize(results, wall)
    s.update({"fp32_bound": fp32_bound, "mode": "sequential: one request at a time, no batching, arrivals "
                                              "ignored (latency = its own set-up and solve)"})
    return s, results


def _max_dE(results, ref_E):
    d = [abs(r.E - ref_E[r.rid]) for r in results if r.rid in ref_E]
    return float(max(d)) if d else None


def run_stream(n_requests: int, rate: float, fp32_bound: float = 0.0, seed: int = 20261203,
               memory_budget: int = None, denserms: float = 1e-6, device: int = 0, workers: int = 4, lanes: int = 4,
               maxiter: int = 100, **stream_kw):
    """Serve one seeded stream; returns (summary dict, results)."""
    reqs = request_stream(n_requests, rate, seed=seed, **stream_kw)
    srv = Server(device=device, memory_budget=memory_budget, fp32_bound=fp32_bound, denserms=denserms,
                 workers=workers, lanes=lanes, maxiter=maxiter)
    try:
        res = srv.serve(reqs, realtime=True)
        s = summarize(res, srv.wall)
        for kind in ("molecule", "qmmm"):
            sub = [r for r in res if r.kind == kind]
            if sub:
                lat = np.array([r.latency for r in sub]) * 1e3
                s[kind] = {"requests": len(sub), "p50_ms": float(np.percentile(lat, 50)),
                           "p99_ms": float(np.percentile(lat, 99)),
                           "mean_iterations": float(np.mean([r.niter for r in sub]))}
        s["host_seconds"] = {k: round(v, 3) for k, v in srv.timers.items()}
        s.update({"rate_per_s": rate, "fp32_bound": fp32_bound, "memory_budget_bytes": srv.budget,
                  "peak_bytes": srv.peak_used, "rejected": len(srv.rejected), "batch_steps": srv.steps,
                  "mean_batch": float(np.mean(srv.batch_sizes)) if srv.batch_sizes else 0.0,
                  "max_batch": int(max(srv.batch_sizes)) if srv.batch_sizes else 0,
                  "warm_starts": int(sum(r.warm for r in res))})
    finally:
        srv.close()
    return s, res


def main(argv=None):
    import argparse
    import json
    ap = argparse.ArgumentParser(description="Serve a seeded stream of RHF requests on one GPU")
    ap.add_argument("--requests", type=int, default=2048)
    ap.add_argument("--rate", type=float, nargs="+", default=[50.0])
    ap.add_argument("--fp32-bound", type=float, default=0.0)
    ap.add_argument("--compare", action="store_true",
                    help="serve each stream in plain FP64 and in the mixed form; report |dE| per request")
    ap.add_argument("--budget-gb", type=float, default=None)
    ap.add_argument("--workers", type=int, default=4, help="set-up threads")
    ap.add_argument("--lanes", type=int, default=4, help="streams the post-build graphs are spread over")
    ap.add_argument("--charges", default="waters", choices=["waters", "independent"],
                    help="QM/MM point charges as rigid TIP3P waters or as independent charges")
    ap.add_argument("--maxiter", type=int, default=100)
    ap.add_argument("--seed", type=int, default=20261203)
    ap.add_argument("--out", default=None)
    ap.add_argument("--warmup", type=int, default=64,
                    help="requests served (untimed) first: module loading, SAD atoms, allocator")
    ap.add_argument("--sequential", action="store_true",
                    help="also solve the stream one request at a time in plain FP64 (no batching): the baseline "
                         "of the served forms' solves/s")
    a = ap.parse_args(argv)
    budget = int(a.budget_gb * (1 << 30)) if a.budget_gb else None
    if a.warmup > 0:
        w = Server(memory_budget=budget, workers=a.workers, lanes=a.lanes, maxiter=a.maxiter)
        w.serve(request_stream(a.warmup, 1000.0, seed=a.seed + 1), realtime=False)
        w.close()
    report = []
    seq = None
    if a.sequential:
        seq, rseq = run_sequential(request_stream(a.requests, 1.0, seed=a.seed, charges=a.charges), maxiter=a.maxiter)
        print(json.dumps({"sequential_fp64": seq}), flush=True)
        report.append({"sequential_fp64": seq})
    for rate in a.rate:
        if a.compare:
            s64, r64 = run_stream(a.requests, rate, 0.0, a.seed, budget, workers=a.workers, lanes=a.lanes,
                                  maxiter=a.maxiter, charges=a.charges)
            bound = a.fp32_bound if a.fp32_bound > 0 else 1e-5
            s32, r32 = run_stream(a.requests, rate, bound, a.seed, budget, workers=a.workers, lanes=a.lanes,
                                  maxiter=a.maxiter, charges=a.charges)
            e64 = {r.rid: r.E for r in r64}
            dE = [abs(r.E - e64[r.rid]) for r in r32 if r.rid in e64]
            s32["max_abs_dE_vs_fp64"] = float(max(dE)) if dE else None
            if seq:
                e_seq = {r.rid: r.E for r in rseq}
                s64["max_abs_dE_vs_sequential_fp64"] = _max_dE(r64, e_seq)
                s32["max_abs_dE_vs_sequential_fp64"] = _max_dE(r32, e_seq)
            line = {"rate_per_s": rate, "fp64": s64, "mixed": s32}
            if seq:
                line["mixed_vs_sequential_fp64"] = s32["solves_per_s"] / seq["solves_per_s"]
                line["fp64_vs_sequential_fp64"] = s64["solves_per_s"] / seq["solves_per_s"]
        else:
            line, res = run_stream(a.requests, rate, a.fp32_bound, a.seed, budget, workers=a.workers, lanes=a.lanes,
                                   maxiter=a.maxiter, charges=a.charges)
            if seq:
                line["vs_sequential_fp64"] = line["solves_per_s"] / seq["solves_per_s"]
        print(json.dumps(line), flush=True)
        report.append(line)

    if a.out:
        with open(a.out, "w") as f:
            json.dump(report, f, indent=1)


if __name__ == "__main__":
    main()
