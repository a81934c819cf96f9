#!/usr/bin/env python
"""Benchmark of the B200 closed-shell two-electron Fock build (QUICK get2e).

Workload (default): 32 water molecules (seed 20261203, 10 Angstrom cube),
RHF/6-31G* with Cartesian d (608 basis functions); one step = one full FP64
Fock build G(D) with integralCutoff 1e-10, primLimit 1e-11, D = the
core-Hamiltonian guess density (idempotent, 320 electrons), synthetic data.

Prints ONE JSON line (rank 0).  ``value`` is Fock builds/s with inputs resident
on the device (CUDA events on the launching stream, L2 flushed between steps);
``e2e`` is the same metric through the host-buffer C ABI (qk_fock2e_host) with
pinned host buffers: the density and o copied in, o + G copied out every step.
``roofline`` is the dominant class kernel against the in-run FP64 FMA peak, its
work counted by the reference-derived model (roofline/flops_per_class.json)
with this library's own operation model beside it.  ``cpu_baseline`` is the C++
oracle (a restatement of the reference's CPU get2e) on a bounded sample.
``reference_gpu`` is QUICK's own CUDA get2e (built from the reference sources by
oracle/Makefile.refgpu) on the same molecule, density and cutoffs.
``workloads`` holds the other named configurations (C40H82/6-31G**,
12 H2O/cc-pVTZ, 4 H2O/STO-3G): builds/s, SCF solves/s and the mixed form.

``--impl reference`` times that CPU implementation alone (all host threads) on
the same workload; under torchrun only rank 0 runs it.  ``--gpus N`` without a
torchrun environment relaunches itself under torchrun with N ranks (replicas).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

INTEGRAL_CUTOFF = 1e-10
PRIM_LIMIT = 1e-11
METRIC = "Fock builds/s (FP64 closed-shell G(D))"
L2_NOTE = "GPU arm: L2 flushed between steps (256 MiB write); CPU arm: n/a"
EXTRA_WORKLOADS = ("c40h82-631gss", "w12-ccpvtz", "w4-sto3g")


def workload(name):
    from quick_b200.basis import build_basis
    from quick_b200 import molecules as M
    if name == "w32-631gs":
        mol, bas = M.water32_631gs()
        desc = "32 H2O (seed 20261203, 10 A cube), RHF/6-31G* (6d)"
    elif name == "w4-sto3g":
        mol, bas = M.water4_sto3g()
        desc = "4 H2O (seed 20261203, 6 A cube), RHF/STO-3G"
    elif name == "c40h82-631gss":
        mol, bas = M.c40h82_631gss()
        desc = "C40H82 all-trans (seed 20261203), RHF/6-31G** (6d)"
    elif name == "w12-ccpvtz":
        mol, bas = M.water12_ccpvtz()
        desc = "12 H2O (seed 20261203, 8 A cube), RHF/cc-pVTZ (Cartesian, f on O)"
    else:
        raise SystemExit(f"unknown workload {name}")
    return build_basis(mol, bas), desc


def bench_config(desc, nbasis, world):
    """The config object of both arms (identical keys and values for one run)."""
    return {"workload": desc, "nbasis": nbasis, "integral_cutoff": INTEGRAL_CUTOFF, "prim_limit": PRIM_LIMIT,
            "density": "core-Hamiltonian guess", "l2": L2_NOTE, "parallelism": f"replicas x{world}"}


def core_guess_density(S, H, nocc):
    w, U = np.linalg.eigh(S)
    X = U[:, w > 1e-8] / np.sqrt(w[w > 1e-8])
    e, C = np.linalg.eigh(X.T @ H @ X)
    C = X @ C[:, :nocc]
    return 2.0 * C @ C.T


def host_cores():
    """(threads this process may use, physical cores among them)."""
    try:
        cpus = sorted(os.sched_getaffinity(0))
    except AttributeError:
        cpus = list(range(os.cpu_count() or 1))
    phys = set()
    try:
        cur = {}
        with open("/proc/cpuinfo") as f:
            for ln in f.read().split("\n\n"):
                kv = dict(x.split(":", 1) for x in ln.splitlines() if ":" in x)
                kv = {k.strip(): v.strip() for k, v in kv.items()}
                if "processor" in kv and int(kv["processor"]) in cpus:
                    cur[int(kv["processor"])] = (kv.get("physical id", "0"), kv.get("core id", kv["processor"]))
        phys = set(cur.values())
    except (OSError, ValueError):
        pass
    return len(cpus), (len(phys) or len(cpus))


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.t:
            self.t.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm),
                "window": "from the first warm-up step to the end of the timed steps"}


def cpu_oracle_sample(basis, D, target_seconds=15.0, nthreads=0):
    """Time the C++ oracle (reference CPU algorithm) on a strided sample of bra
    shells.  Returns (builds/s extrapolated, description, seconds, stride, G or
    None): G is the full oracle Fock matrix when the sample was the whole loop."""
    from oracle import oracle as O
    orc = O.Oracle(basis)
    Y, cp = orc.schwarz(nthreads)
    cm = orc.density_cutoff(D)
    ns = basis.nshell
    stride = max(1, ns // 4)
    G = None
    while True:
        t0 = time.perf_counter()
        G, _ = orc.get2e(D, cm, Y, cp, INTEGRAL_CUTOFF, PRIM_LIMIT, ii_stride=stride, nthreads=nthreads)
        t = time.perf_counter() - t0
        if t * 2.5 > target_seconds or stride == 1:
            break
        stride = max(1, stride // 2)
    rate = 1.0 / (t * stride)
    desc = (f"bra shells II = 0, {stride}, {2 * stride}, ... (1/{stride} of the quartet loop, "
            f"{t:.1f} s), extrapolated x{stride}; oracle built for {O.host_isa()}")
    return rate, desc, t, stride, (G if stride == 1 else None)


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    world = int(os.environ.get("WORLD_SIZE", str(args.gpus)))
    basis, desc = workload(args.workload)
    S, T, V = O.oei(basis)
    D = core_guess_density(S, T + V, basis.mol.nelec // 2)
    orc = O.Oracle(basis)
    Y, cp = orc.schwarz(0)
    cm = orc.density_cutoff(D)
    ns = basis.nshell
    # size the per-step sample to a few seconds of CPU work
    stride = max(1, ns // 4)
    while True:
        t0 = time.perf_counter()
        orc.get2e(D, cm, Y, cp, INTEGRAL_CUTOFF, PRIM_LIMIT, ii_stride=stride)
        t = time.perf_counter() - t0
        if t * 2.0 > args.ref_step_seconds or stride == 1:
            break
        stride = max(1, stride // 2)
    for _ in range(max(0, args.warmup - 1)):
        orc.get2e(D, cm, Y, cp, INTEGRAL_CUTOFF, PRIM_LIMIT, ii_stride=stride)
    times = []
    for k in range(args.steps):
        off = k % stride
        t0 = time.perf_counter()
        orc.get2e(D, cm, Y, cp, INTEGRAL_CUTOFF, PRIM_LIMIT, ii_range=(off, 0), ii_stride=stride)
        times.append((time.perf_counter() - t0) * stride)
    ms = 1000.0 * statistics.mean(times)
    value = 1000.0 / ms
    threads, cores = host_cores()
    sample = (f"each step: bra shells II = k mod {stride}, k + {stride}, ... (1/{stride} of the quartet loop), "
              f"time x{stride}; {threads} threads on {cores} physical cores; oracle built for {O.host_isa()}")
    line = {
        "impl": "reference", "metric": METRIC, "value": value,
        "unit": "builds/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": bench_config(desc, basis.nbasis, world),
        "cpu_baseline": {"value": value, "unit": "builds/s", "cores": cores, "threads": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "builds/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def max_over_ranks(x: float, pg, device) -> float:
    """The largest of every rank's x (the job's time is its slowest rank's); x
    itself without a process group.  Every rank must call it at the same point."""
    if not pg:
        return float(x)
    import torch
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def reference_model():
    path = os.path.join(ROOT, "roofline", "flops_per_class.json")
    try:
        return json.load(open(path))["classes"]
    except (OSError, ValueError, KeyError):
        return None


def class_figures(eng, D, o, stream, flush, nprof):
    """Per class: kernel time alone (CUDA events, classes serialised, mean of
    ``nprof`` builds), quartets and primitive quartets listed and evaluated, this
    library's operation model."""
    import ctypes
    import torch
    from quick_b200._native import lib
    L = lib()
    h = ctypes.c_void_p(eng.h)
    ncls = 64
    P = lambda a: ctypes.c_void_p(a.ctypes.data)  # noqa: E731
    cls = np.zeros(4 * ncls, dtype=np.int32)
    ms_tot = np.zeros(ncls)
    ms_buf = np.zeros(ncls, dtype=np.float32)
    L.qk_set_profiling(h, 1, 0)
    for _ in range(nprof):
        flush.fill_(1.0)
        o.zero_()
        eng.fock2e(D, o=o, stream=stream)
        nc = L.qk_class_profile(h, ncls, P(cls), P(ms_buf), None, None, None, None, None, None)
        ms_tot[:nc] += ms_buf[:nc]
    L.qk_set_profiling(h, 0, 1)
    o.zero_()
    eng.fock2e(D, o=o)
    torch.cuda.synchronize()
    ql, pql, qd, pqd = (np.zeros(ncls, dtype=np.int64) for _ in range(4))
    pf, qf = np.zeros(ncls), np.zeros(ncls)
    nc = L.qk_class_profile(h, ncls, P(cls), None, P(ql), P(pql), P(qd), P(pqd), P(pf), P(qf))
    L.qk_set_profiling(h, 0, 0)
    out = []
    for i in range(nc):
        if ql[i] == 0:
            continue
        out.append({"tag": "".join("spdf"[x] for x in cls[4 * i:4 * i + 4]),
                    "L": [int(x) for x in cls[4 * i:4 * i + 4]], "ms": float(ms_tot[i] / nprof),
                    "q_listed": int(ql[i]), "pq_listed": int(pql[i]), "q_done": int(qd[i]),
                    "pq_done": int(pqd[i]), "own_prim": float(pf[i]), "own_quartet": float(qf[i])})
    return out


def roofline_from(classes, peak_tf, ms_build, traffic_table, wl):
    """Roofline of the dominant class kernel (by time alone) with the work counted
    by the reference-derived model, and the same with this library's model.
    Work in GFLOP, times in ms: GFLOP / ms = TFLOP/s."""
    ref = reference_model()
    tot_ms = sum(c["ms"] for c in classes) or 1e-30
    for c in classes:
        c["own_gflop"] = (c["pq_done"] * c["own_prim"] + c["q_done"] * c["own_quartet"]) * 1e-9
        r = ref.get(c["tag"]) if ref else None
        c["ref_gflop"] = ((c["pq_done"] * r["prim"] + c["q_done"] * r["quartet"]) * 1e-9) if r else None
    top = max(classes, key=lambda c: c["ms"])
    ach_ref = top["ref_gflop"] / top["ms"] if top["ref_gflop"] is not None and top["ms"] > 0 else None
    ach_own = top["own_gflop"] / top["ms"] if top["ms"] > 0 else 0.0
    traffic = None
    if traffic_table:
        traffic = traffic_table.get(wl, {}).get(top["tag"])
    all_ref = sum(c["ref_gflop"] or 0.0 for c in classes)
    all_own = sum(c["own_gflop"] for c in classes)
    return {
        "bound": "fp64", "kernel": f"class kernel <{','.join(str(x) for x in top['L'])}> ({top['tag']})",
        "achieved": round(ach_ref, 4) if ach_ref is not None else None, "peak": round(peak_tf, 4),
        "unit": "TFLOP/s", "frac": round(ach_ref / peak_tf, 4) if ach_ref is not None and peak_tf > 0 else None,
        "traffic": traffic,
        "work_model": "reference-derived operation counts (roofline/flops_per_class.json, counted from QUICK's "
                      "generated VRR blocks, gpu_fmt.h, hrr.f90 and eri.fh) x the quartets and primitive quartets "
                      "the kernel evaluated after screening",
        "achieved_own_model": round(ach_own, 4),
        "frac_own_model": round(ach_own / peak_tf, 4) if peak_tf > 0 else None,
        "peak_source": "measured in-run: FP64 FMA probe kernel (qk_fp64_peak); MEASURED_PEAKS.json has no FP64 "
                       "figure",
        "share_of_build": round(top["ms"] / tot_ms, 4),
        "all_classes_tflops": round(all_ref / ms_build, 4) if ms_build > 0 else None,
        "all_classes_tflops_own_model": round(all_own / ms_build, 4) if ms_build > 0 else None,
        "timing": "dominant class kernel timed alone with CUDA events on its launching stream; all_classes uses "
                  "the whole build's time",
    }


def time_builds(eng, D, o, stream, flush, steps):
    import torch
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    out = []
    for _ in range(steps):
        flush.fill_(1.0)           # L2 flush (256 MiB write) outside the timed window
        o.zero_()
        ev0.record(stream)
        eng.fock2e(D, o=o, stream=stream)
        ev1.record(stream)
        ev1.synchronize()
        out.append(ev0.elapsed_time(ev1))
    return out


def reference_gpu_figures(basis, D_host, steps):
    """QUICK's own CUDA get2e on the same molecule, density and cutoffs (its own
    process), or a reason why not."""
    try:
        from oracle import oracle as O
        from oracle import refgpu
    except Exception as e:  # noqa: BLE001
        return {"unavailable": f"import failed: {e}"}
    if not refgpu.available():
        return {"unavailable": "oracle/_ref/refgpu_get2e not built (make -f oracle/Makefile.refgpu REF=...)"}
    if basis.has_f:
        return {"unavailable": "the reference's f-enabled GPU get2e (-DGPU_SPDF) does not finish compiling "
                               "(ptxas > 1 h); only its s/p/d build exists here"}
    orc = O.Oracle(basis)
    Y, cp = orc.schwarz()
    cm = orc.density_cutoff(D_host)
    try:
        G, info = refgpu.run(basis, D_host, cm, Y, cp, INTEGRAL_CUTOFF, PRIM_LIMIT, steps=steps, warmup=2)
    except Exception as e:  # noqa: BLE001
        return {"unavailable": f"harness failed: {str(e)[-300:]}"}
    kern = info["kernel_ms_mean"]
    call = info["call_ms_mean"]
    return {"value": 1000.0 / kern if kern > 0 else None, "unit": "builds/s", "ms_per_step": kern,
            "call_builds_per_s": 1000.0 / call if call > 0 else None, "call_ms_per_step": call,
            "setup_s": info["setup_s"], "bit_identical_repeat": info["bit_identical_repeat"],
            "what": "QUICK's own get2e kernels (src/gpu/cuda/gpu_get2e.cu:594-637, built for sm_100 with the "
                    "reference's flags) timed alone with CUDA events, L2 flushed; call_* = its whole per-build "
                    "call sequence gpu_upload_calculated_ + gpu_upload_cutoff_ + gpu_get_cshell_eri_ (host "
                    "clock, host buffers)", "G": G}


def measure(name, args, dev, stream, flush, local, world, pg, full):
    """All figures of one workload.  ``full``: the headline workload (more steps,
    the CPU baseline and the parity check against the oracle)."""
    import torch
    from quick_b200.get2e import Get2e
    from quick_b200.scf import RHF, GraphSCF, oei
    basis, desc = workload(name)
    n = basis.nbasis
    S, T, V = oei(basis, device=local)
    D_host = core_guess_density(S, T + V, basis.mol.nelec // 2)
    eng = Get2e(basis, device=local, integral_cutoff=INTEGRAL_CUTOFF, prim_limit=PRIM_LIMIT)
    D = torch.tensor(D_host, device=dev)
    o = torch.zeros((n, n), dtype=torch.float64, device=dev)
    steps = args.steps if full else max(5, args.steps // 2)
    res = {"workload": desc, "nbasis": n}

    clocks = ClockSampler(local) if full else None
    if clocks:
        if pg:
            pg.barrier()
        clocks.start()
    for _ in range(args.warmup):           # the first build also builds the tables and work lists
        o.zero_()
        eng.fock2e(D, o=o)
    torch.cuda.synchronize()
    tune_report = None
    if not args.no_tune:                   # launch shapes tuned on this molecule before timing
        from quick_b200 import autotune
        tune_report = autotune.tune(eng, D)
        for _ in range(args.warmup):
            o.zero_()
            eng.fock2e(D, o=o)
        torch.cuda.synchronize()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    step_ms = time_builds(eng, D, o, stream, flush, steps)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    clk = clocks.stop() if clocks else None
    total_ms = max_over_ranks(float(sum(step_ms)), pg, dev)
    ms_per_step = total_ms / steps
    G_dev = o.cpu().numpy()
    res.update({"value": world * 1000.0 / ms_per_step, "ms_per_step": ms_per_step, "steps": steps,
                "p50_ms": float(np.percentile(step_ms, 50)), "p99_ms": float(np.percentile(step_ms, 99)),
                "launches_per_build": int(eng.work()["launches"]), "clocks": clk})

    from quick_b200._native import lib
    import ctypes
    peak = ctypes.c_double(0.0)
    lib().qk_fp64_peak(local, ctypes.byref(peak))
    peak_tf = peak.value * 1e-3
    classes = class_figures(eng, D, o, stream, flush, max(3, min(steps, 10)))
    traffic_table = None
    try:
        traffic_table = json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))
    except (OSError, ValueError):
        pass
    res["roofline"] = roofline_from(classes, peak_tf, ms_per_step, traffic_table, name)
    res["classes"] = {c["tag"]: {"ms_alone": round(c["ms"], 4), "quartets": c["q_done"],
                                 "prim_quartets": c["pq_done"], "quartets_listed": c["q_listed"],
                                 "tflops_ref_model": round(c["ref_gflop"] / c["ms"], 3)
                                 if c["ref_gflop"] is not None and c["ms"] > 0 else None,
                                 "tflops_own_model": round(c["own_gflop"] / c["ms"], 3) if c["ms"] > 0 else None}
                      for c in classes}

    # end to end through the host-buffer C ABI: pinned D and o in, o + G out, every step
    Dp = torch.tensor(D_host).pin_memory()
    op = torch.zeros((n, n), dtype=torch.float64).pin_memory()
    Dn, on = Dp.numpy(), op.numpy()
    for _ in range(2):
        eng.fock2e_host(Dn, o=on)
    if pg:
        pg.barrier()
    e2e_t = []
    for _ in range(steps):
        on[:] = 0.0   # the caller's fresh output buffer; the timed region is the API call
        t0 = time.perf_counter()
        r_host = eng.fock2e_host(Dn, o=on)
        e2e_t.append(time.perf_counter() - t0)
    e2e_total = max_over_ranks(float(sum(e2e_t)), pg, dev)
    res["e2e"] = {"value": world * steps / e2e_total, "unit": "builds/s", "h2d_bytes_per_step": 16 * n * n,
                  "d2h_bytes_per_step": 8 * n * n}
    res["bit_identical_host_vs_device"] = bool(np.array_equal(G_dev, r_host))

    # mixed form: FP32 vertical recursion below a Schwarz bound product
    G_mixed = None
    if args.fp32_bound > 0:
        eng.set_precision(args.fp32_bound)
        for _ in range(2):
            o.zero_()
            eng.fock2e(D, o=o, stream=stream)
        torch.cuda.synchronize()
        mixed_ms = time_builds(eng, D, o, stream, flush, steps)
        G_mixed = o.cpu().numpy()
        nq32 = eng.fp32_quartets()
        eng.set_precision(0.0)
        mms = float(np.mean(mixed_ms))
        res["mixed"] = {"fp32_bound": args.fp32_bound, "builds_per_s": world * 1000.0 / mms, "ms_per_step": mms,
                        "speedup_vs_fp64": ms_per_step / mms,
                        "max_abs_dG_vs_fp64_gpu": float(np.abs(G_mixed - G_dev).max()),
                        "fp32_quartet_fraction": nq32 / max(1, sum(c["q_listed"] for c in classes))}

    if not args.no_scf:
        def median_run(run, k):
            runs = sorted((run() for _ in range(k)), key=lambda x: x["seconds"])
            return runs[len(runs) // 2]
        k = 3 if full else 1
        rhf = RHF(basis, device=local, engine=eng)
        rhf.run(denserms=1e-7, guess="sad")
        r2 = median_run(lambda: rhf.run(denserms=1e-7, guess="sad"), k)
        gs = GraphSCF(RHF(basis, device=local, engine=eng))
        gs.run(denserms=1e-7, guess="sad")    # the first run captures the graph
        g2 = median_run(lambda: gs.run(denserms=1e-7, guess="sad"), k)
        graph_rate, eager_rate = 1.0 / g2["seconds"], 1.0 / r2["seconds"]
        best = g2 if graph_rate >= eager_rate else r2
        scf = {"solves_per_s": round(max(graph_rate, eager_rate), 4), "seconds": round(best["seconds"], 3),
               "iterations": best["niter"], "E": best["E"], "converged": bool(best["converged"]),
               "denserms": 1e-7, "incremental_builds": True, "guess": "SAD",
               "path": ("one CUDA graph per SCF cycle (Fock build, DIIS, SP2 density)" if best is g2
                        else "eager cycle (torch eigh per cycle)"),
               "graph_sp2": {"solves_per_s": round(graph_rate, 4), "iterations": g2["niter"], "E": g2["E"],
                             "sp2_steps": g2["sp2_steps"]},
               "eager_eigh": {"solves_per_s": round(eager_rate, 4), "iterations": r2["niter"], "E": r2["E"]},
               "abs_dE_graph_vs_eager": abs(g2["E"] - r2["E"])}
        if "mixed" in res:
            eng.set_precision(args.fp32_bound)
            gm = GraphSCF(RHF(basis, device=local, engine=eng))
            gm.run(denserms=1e-7, guess="sad")
            r3 = gm.run(denserms=1e-7, guess="sad")
            eng.set_precision(0.0)
            h64 = {it: e for it, e, _ in g2["history"]}
            per_it = [abs(e - h64[it]) for it, e, _ in r3["history"] if it in h64]
            res["mixed"]["scf"] = {"solves_per_s": round(1.0 / r3["seconds"], 4), "iterations": r3["niter"],
                                   "E": r3["E"], "abs_dE_vs_fp64_gpu": abs(r3["E"] - g2["E"]),
                                   "max_abs_dE_per_iteration_vs_fp64_gpu": max(per_it) if per_it else None,
                                   "abs_dE_per_iteration_vs_fp64_gpu": per_it,
                                   "converged": bool(r3["converged"])}
        res["scf"] = scf

    # The baselines leg (headline workload, one rank): the reference implementations
    # timed beside this one -- the CPU get2e restatement on the host cores and
    # QUICK's own CUDA get2e on this GPU -- and this run's G against the oracle's.
    # The only part of the GPU arm that runs anything under oracle/.
    if full and not args.no_cpu and world == 1 and args.reference_gpu:
        ref = reference_gpu_figures(basis, D_host, steps)
        G_ref = ref.pop("G", None)
        if G_ref is not None:
            ref["max_abs_dG_vs_ours"] = float(np.abs(G_ref - G_dev).max())
            ref["speedup_ours_vs_reference_gpu"] = res["value"] / world / ref["value"] if ref.get("value") else None
            ref["e2e_speedup_ours_vs_reference_gpu_call"] = (
                res["e2e"]["value"] / world / ref["call_builds_per_s"] if ref.get("call_builds_per_s") else None)
        res["reference_gpu"] = ref

    if full and not args.no_cpu and world == 1:
        rate, sdesc, t, stride, G_orc = cpu_oracle_sample(basis, D_host, args.cpu_seconds)
        threads, cores = host_cores()
        res["cpu_baseline"] = {"value": rate, "unit": "builds/s", "cores": cores, "threads": threads, "kind": "port",
                               "sample": sdesc}
        if G_orc is not None:
            res["parity_vs_oracle"] = {"max_abs_dG_fp64": float(np.abs(G_dev - G_orc).max()),
                                       "max_abs_dG_mixed": float(np.abs(G_mixed - G_orc).max())
                                       if G_mixed is not None else None,
                                       "what": "this run's timed G (and the mixed form's) against the oracle's "
                                               "full G on the same density and cutoffs"}
    if tune_report is not None:
        res["autotune"] = {"ms_default": round(tune_report["ms_default"], 4),
                           "ms_tuned": round(tune_report["ms_tuned"], 4),
                           "best_streams": tune_report["best_streams"], "merge_sp": tune_report["merge_sp"]}
    eng.close()
    return res


SERVE_RATE = 200.0
SERVE_SEED = 20261203
SERVE_BOUND = 1e-5


def serving_figures(args, baselines):
    """The served form on a short seeded stream (requests of 1-40 waters in STO-3G
    or 6-31G*, a quarter QM/MM repeats with 4000 point charges, Poisson arrivals at
    SERVE_RATE): the mixed form served with continuous batching against the plain
    FP64 path solving the same requests one at a time (``run_sequential``), with
    |dE| per request against the sequential FP64 energies and, in the baselines
    leg, against the oracle's SCF on a sample of the requests."""
    from quick_b200.serve import Server, request_stream, run_sequential, run_stream, _max_dE
    w = Server(workers=args.serve_workers)
    w.serve(request_stream(32, 1000.0, seed=SERVE_SEED + 1), realtime=False)
    w.close()
    n = args.serve_requests
    seq, rseq = run_sequential(request_stream(n, 1.0, seed=SERVE_SEED))
    served, rsrv = run_stream(n, SERVE_RATE, SERVE_BOUND, SERVE_SEED, workers=args.serve_workers,
                              lanes=args.serve_lanes)
    e_seq = {r.rid: r.E for r in rseq}
    out = {"requests": n, "rate_per_s": SERVE_RATE, "fp32_bound": SERVE_BOUND, "workers": args.serve_workers,
           "lanes": args.serve_lanes,
           "served_mixed": {k: served[k] for k in ("solves_per_s", "p50_ms", "p99_ms", "mean_iterations", "converged",
                                                   "mean_batch", "max_batch", "peak_bytes", "molecule", "qmmm")
                            if k in served},
           "sequential_fp64": {k: seq[k] for k in ("solves_per_s", "p50_ms", "p99_ms", "mean_iterations", "converged")},
           "served_over_sequential": served["solves_per_s"] / seq["solves_per_s"],
           "max_abs_dE_served_mixed_vs_sequential_fp64": _max_dE(rsrv, e_seq),
           "stream": "seeded: Poisson arrivals; 1-40 waters log-uniform, basis uniform over {STO-3G, 6-31G*}; "
                     "25% QM/MM repeats (20-water QM region, 4000 TIP3P point charges, warm start)"}
    if baselines:
        # the oracle's RHF (same cutoffs, tight convergence) on a sample of the requests:
        # the smallest molecule requests of each basis and the first QM/MM request
        from oracle import oracle as O
        from quick_b200.basis import build_basis
        reqs = {r.rid: r for r in request_stream(n, 1.0, seed=SERVE_SEED)}
        got = {r.rid: r for r in rsrv}
        mols = sorted((r for r in reqs.values() if r.kind == "molecule"), key=lambda r: (len(r.mol.Z), r.rid))
        pick = [r for b in ("STO-3G", "6-31G*") for r in [x for x in mols if x.basis == b][:2]]
        pick += [r for r in reqs.values() if r.kind == "qmmm"][:1]
        rows = []
        t0 = time.perf_counter()
        for r in pick:
            b = build_basis(r.mol, r.basis)
            ref = O.rhf(b, integral_cutoff=1e-10, prim_limit=1e-11, conv=1e-8, ext_charges=r.ext_charges)
            rows.append({"rid": r.rid, "kind": r.kind, "basis": r.basis, "nbasis": b.nbasis,
                         "abs_dE_served_mixed_vs_oracle": abs(got[r.rid].E - ref["E"]),
                         "abs_dE_sequential_fp64_vs_oracle": abs(e_seq[r.rid] - ref["E"])})
        out["vs_oracle"] = {"sample": rows, "max_abs_dE_served_mixed": max(x["abs_dE_served_mixed_vs_oracle"]
                                                                          for x in rows),
                            "oracle_seconds": round(time.perf_counter() - t0, 1)}
    return out


def run_ours(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    head = measure(args.workload, args, dev, stream, flush, local, world, pg, full=True)
    extras = {}
    if not args.no_extra:
        for wl in [w for w in EXTRA_WORKLOADS if w != args.workload]:
            extras[wl] = measure(wl, args, dev, stream, flush, local, world, pg, full=False)
    serving = None
    if not args.no_serve and world == 1:
        del flush
        torch.cuda.empty_cache()
        serving = serving_figures(args, baselines=not args.no_cpu)

    if rank == 0:
        line = {
            "metric": METRIC, "value": head["value"], "unit": "builds/s", "n_gpus": world, "steps": head["steps"],
            "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "p50_ms": head["p50_ms"],
            "p99_ms": head["p99_ms"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": bench_config(head["workload"], head["nbasis"], world),
            "roofline": head["roofline"], "cpu_baseline": head.get("cpu_baseline"), "e2e": head["e2e"],
            "gpu_launches": head["launches_per_build"] * head["steps"], "clocks": head["clocks"],
            "reference_gpu": head.get("reference_gpu"), "parity_vs_oracle": head.get("parity_vs_oracle"),
            "scf": head.get("scf"), "mixed": head.get("mixed"),
            "bit_identical_host_vs_device": head["bit_identical_host_vs_device"], "classes": head["classes"],
            "autotune": head.get("autotune"), "serving": serving,
            "workloads": {k: {kk: v[kk] for kk in ("workload", "nbasis", "value", "ms_per_step", "e2e", "scf", "mixed",
                                                   "roofline", "launches_per_build") if kk in v}
                          for k, v in extras.items()},
        }
        print(json.dumps(line), flush=True)
    if pg:
        pg.destroy_process_group()


def relaunch_under_torchrun(args):
    """``--gpus N`` (N > 1) outside torchrun: start N ranks of this script."""
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__), *sys.argv[1:]]
    return subprocess.call(cmd)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="w32-631gs")
    ap.add_argument("--no-scf", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="only the headline workload")
    ap.add_argument("--no-reference-gpu", dest="reference_gpu", action="store_false",
                    help="skip QUICK's own GPU get2e on the headline workload")
    ap.add_argument("--fp32-bound", type=float, default=1e-5,
                    help="mixed form: FP32 below this Schwarz bound product (0 = skip)")
    ap.add_argument("--no-cpu", action="store_true",
                    help="skip the baselines leg (CPU oracle sample, QUICK's GPU get2e, parity vs the oracle)")
    ap.add_argument("--no-tune", action="store_true", help="default launch shapes (no autotuning)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-serve", action="store_true", help="skip the serving leg (1 GPU only)")
    ap.add_argument("--serve-requests", type=int, default=1024)
    ap.add_argument("--serve-workers", type=int, default=8)
    ap.add_argument("--serve-lanes", type=int, default=4)
    ap.add_argument("--ref-step-seconds", type=float, default=6.0)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(relaunch_under_torchrun(args))
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
