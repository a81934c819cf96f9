#!/usr/bin/env python
"""Benchmark of the B200 closed-shell two-electron Fock build (QUICK get2e).

Workload (default): 32 water molecules (seed 20261203, 10 Angstrom cube),
RHF/6-31G* with Cartesian d (608 basis functions); one step = one full FP64
Fock build G(D) with integralCutoff 1e-10, primLimit 1e-11, D = the
core-Hamiltonian guess density (idempotent, 320 electrons), synthetic data.

Prints ONE JSON line (rank 0).  ``value`` is Fock builds/s with inputs resident
on the device (CUDA events on the launching stream, L2 flushed between steps);
``e2e`` is the same metric through the host-buffer C ABI (qk_fock2e_host) with
pinned host buffers: the density and o copied in, o + G copied out every step.  ``roofline`` is the
dominant class kernel against the in-run FP64 FMA peak.  ``cpu_baseline`` is the
C++ oracle (a restatement of the reference's CPU get2e) on a bounded sample.

``--impl reference`` times that CPU implementation alone (all host threads) on
the same workload; under torchrun only rank 0 runs it.
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


def core_guess_density(S, H, nocc):
    w, U = np.linalg.eigh(S)
    X = U[:, w > 1e-8] / np.sqrt(w[w > 1e-8])
    e, C = np.linalg.eigh(X.T @ H @ X)
    C = X @ C[:, :nocc]
    return 2.0 * C @ C.T


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
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
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
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_oracle_sample(basis, D, target_seconds=15.0, nthreads=0):
    """Time the C++ oracle (reference CPU algorithm) on a strided sample of bra
    shells; returns (builds/s extrapolated, description, threads)."""
    from oracle import oracle as O
    orc = O.Oracle(basis)
    Y, cp = orc.schwarz(nthreads)
    cm = orc.density_cutoff(D)
    ns = basis.nshell
    stride = max(1, ns // 4)
    t = 0.0
    while True:
        t0 = time.perf_counter()
        orc.get2e(D, cm, Y, cp, INTEGRAL_CUTOFF, PRIM_LIMIT, ii_stride=stride, nthreads=nthreads)
        t = time.perf_counter() - t0
        if t * 2.5 > target_seconds or stride == 1:
            break
        stride = max(1, stride // 2)
    threads = nthreads if nthreads > 0 else (os.cpu_count() or 1)
    rate = 1.0 / (t * stride)
    desc = (f"bra shells II = 0, {stride}, {2 * stride}, ... (1/{stride} of the quartet loop, "
            f"{t:.1f} s), extrapolated x{stride}")
    return rate, desc, threads, t, stride


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    basis, desc = workload(args.workload)
    S, T, V = O.oei(basis)
    D = core_guess_density(S, T + V, basis.mol.nelec // 2)
    from oracle import oracle as O2
    orc = O2.Oracle(basis)
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
    threads = os.cpu_count() or 1
    sample = (f"each step: bra shells II = k mod {stride}, k + {stride}, ... (1/{stride} of the quartet loop), "
              f"time x{stride}")
    line = {
        "impl": "reference", "metric": "Fock builds/s (FP64 closed-shell G(D))", "value": value,
        "unit": "builds/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": desc, "nbasis": basis.nbasis, "integral_cutoff": INTEGRAL_CUTOFF,
                   "prim_limit": PRIM_LIMIT, "density": "core-Hamiltonian guess"},
        "cpu_baseline": {"value": value, "unit": "builds/s", "cores": threads, "kind": "port", "sample": sample},
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
    from quick_b200 import _native
    from quick_b200.get2e import Get2e
    from quick_b200.scf import RHF, oei
    import ctypes

    basis, desc = workload(args.workload)
    n = basis.nbasis
    S, T, V = oei(basis, device=local)
    D_host = core_guess_density(S, T + V, basis.mol.nelec // 2)
    eng = Get2e(basis, device=local, integral_cutoff=INTEGRAL_CUTOFF, prim_limit=PRIM_LIMIT)
    L = _native.lib()
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    D = torch.tensor(D_host, device=dev)
    o = torch.zeros((n, n), dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    # warm-up (first build also builds the pair tables and work lists)
    for _ in range(args.warmup):
        o.zero_()
        eng.fock2e(D, o=o)
    torch.cuda.synchronize()
    # launch shapes tuned on this molecule before the timed region (quick_b200.autotune)
    tune_report = None
    if not args.no_tune:
        from quick_b200 import autotune
        tune_report = autotune.tune(eng, D)
        for _ in range(args.warmup):
            o.zero_()
            eng.fock2e(D, o=o)
        torch.cuda.synchronize()
    launches = L.qk_launches_per_build(ctypes.c_void_p(eng.h))
    ncls = 64
    cls = np.zeros(4 * ncls, dtype=np.int32)
    cls_ms_total = np.zeros(ncls, dtype=np.float64)
    ms_buf = np.zeros(ncls, dtype=np.float32)
    P = lambda a: ctypes.c_void_p(a.ctypes.data)  # noqa: E731

    clocks = ClockSampler(local)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    clocks.start()
    step_ms = []
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    for _ in range(args.steps):
        flush.fill_(1.0)           # L2 flush (256 MiB write) outside the timed window
        o.zero_()
        ev0.record(stream)
        eng.fock2e(D, o=o, stream=stream)
        ev1.record(stream)
        ev1.synchronize()
        step_ms.append(ev0.elapsed_time(ev1))
    torch.cuda.synchronize()
    clk = clocks.stop()
    total_ms = float(sum(step_ms))
    total_ms = max_over_ranks(total_ms, pg, dev)
    ms_per_step = total_ms / args.steps
    value = world * 1000.0 / ms_per_step

    # per-class kernel time: the same builds with every class kernel timed alone
    # (CUDA events on the launching stream; classes serialised in this pass)
    L.qk_set_profiling(ctypes.c_void_p(eng.h), 1, 0)
    nprof = max(3, min(args.steps, 10))
    for _ in range(nprof):
        flush.fill_(1.0)
        o.zero_()
        eng.fock2e(D, o=o, stream=stream)
        nc = L.qk_class_profile(ctypes.c_void_p(eng.h), ncls, P(cls), P(ms_buf), None, None, None, None, None, None)
        cls_ms_total[:nc] += ms_buf[:nc]
    L.qk_set_profiling(ctypes.c_void_p(eng.h), 0, 0)

    # work counters of one build (deterministic; not timed)
    L.qk_set_profiling(ctypes.c_void_p(eng.h), 0, 1)
    o.zero_()
    eng.fock2e(D, o=o)
    torch.cuda.synchronize()
    ql = np.zeros(ncls, dtype=np.int64)
    pql = np.zeros(ncls, dtype=np.int64)
    qd = np.zeros(ncls, dtype=np.int64)
    pqd = np.zeros(ncls, dtype=np.int64)
    pf = np.zeros(ncls)
    qf = np.zeros(ncls)
    nc = L.qk_class_profile(ctypes.c_void_p(eng.h), ncls, P(cls), None, P(ql), P(pql), P(qd), P(pqd), P(pf), P(qf))
    L.qk_set_profiling(ctypes.c_void_p(eng.h), 0, 0)
    flops = pqd[:nc] * pf[:nc] + qd[:nc] * qf[:nc]
    cls_ms = cls_ms_total[:nc] / nprof
    top = int(np.argmax(cls_ms))
    peak = ctypes.c_double(0.0)
    L.qk_fp64_peak(local, ctypes.byref(peak))
    peak_tf = peak.value * 1e-3
    top_tf = flops[top] / (cls_ms[top] * 1e-3) * 1e-12 if cls_ms[top] > 0 else 0.0
    all_tf = float(flops.sum()) / (ms_per_step * 1e-3) * 1e-12
    tag = "".join("spdf"[x] for x in cls[4 * top:4 * top + 4])
    traffic = None
    prof_path = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(prof_path):
        try:
            traffic = json.load(open(prof_path)).get(args.workload, {}).get(tag)
        except Exception:
            traffic = None
    per_class = {
        "".join("spdf"[x] for x in cls[4 * i:4 * i + 4]): {
            "ms_alone": round(float(cls_ms[i]), 4),
            "share_alone": round(float(cls_ms[i] / max(cls_ms.sum(), 1e-30)), 4),
            "quartets": int(qd[i]), "prim_quartets": int(pqd[i]),
            "quartets_listed": int(ql[i]), "prim_quartets_listed": int(pql[i]),
            "tflops": round(float(flops[i] / (cls_ms[i] * 1e-3) * 1e-12) if cls_ms[i] > 0 else 0.0, 3)}
        for i in range(nc) if ql[i] > 0}

    # end to end through the host-buffer C ABI: pinned D in, G out, every step
    Dp = torch.tensor(D_host).pin_memory()
    op = torch.zeros((n, n), dtype=torch.float64).pin_memory()
    Dn = Dp.numpy()
    on = op.numpy()
    for _ in range(2):
        eng.fock2e_host(Dn, o=on)
    if pg:
        pg.barrier()
    e2e_t = []
    for _ in range(args.steps):
        on[:] = 0.0   # the caller's fresh output buffer; the timed region is the API call
        t0 = time.perf_counter()
        res = eng.fock2e_host(Dn, o=on)
        e2e_t.append(time.perf_counter() - t0)
    e2e_total = max_over_ranks(float(sum(e2e_t)), pg, dev)
    e2e_value = world * args.steps / e2e_total
    # parity spot check of the timed result (bitwise run-to-run identity)
    G_dev = o.cpu().numpy()
    bit_identical = bool(np.array_equal(G_dev, res))

    # mixed form: FP32 vertical recursion below a Schwarz bound product
    mixed = None
    if args.fp32_bound > 0:
        eng.set_precision(args.fp32_bound)
        for _ in range(2):
            o.zero_()
            eng.fock2e(D, o=o, stream=stream)
        torch.cuda.synchronize()
        mixed_ms = []
        for _ in range(args.steps):
            flush.fill_(1.0)
            o.zero_()
            ev0.record(stream)
            eng.fock2e(D, o=o, stream=stream)
            ev1.record(stream)
            ev1.synchronize()
            mixed_ms.append(ev0.elapsed_time(ev1))
        G_mixed = o.cpu().numpy()
        nq32 = eng.fp32_quartets()
        eng.set_precision(0.0)
        mms = float(np.mean(mixed_ms))
        mixed = {"fp32_bound": args.fp32_bound, "builds_per_s": world * 1000.0 / mms, "ms_per_step": mms,
                 "speedup_vs_fp64": ms_per_step / mms,
                 "max_abs_dF_vs_fp64": float(np.abs(G_mixed - G_dev).max()),
                 "fp32_quartet_fraction": nq32 / max(1, int(ql[:nc].sum()))}

    scf = None
    if not args.no_scf:
        from quick_b200.scf import GraphSCF
        # eager loop (torch eigh per cycle), then the graph-captured iteration (SP2 density)
        # each path: one untimed solve, then the median of three timed solves
        def median_run(run):
            runs = sorted((run() for _ in range(3)), key=lambda x: x["seconds"])
            return runs[1]
        rhf = RHF(basis, device=local, engine=eng)
        rhf.run(denserms=1e-7, guess="sad")
        r2 = median_run(lambda: rhf.run(denserms=1e-7, guess="sad"))
        gs = GraphSCF(RHF(basis, device=local, engine=eng))
        gs.run(denserms=1e-7, guess="sad")    # first run captures the graph
        g2 = median_run(lambda: gs.run(denserms=1e-7, guess="sad"))
        # headline: the faster of the two paths on this molecule (eigh wins on tiny ones,
        # where SP2's fixed number of small GEMMs costs more than one eigh)
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
        if mixed is not None:
            eng.set_precision(args.fp32_bound)
            gm = GraphSCF(RHF(basis, device=local, engine=eng))
            gm.run(denserms=1e-7, guess="sad")
            r3 = gm.run(denserms=1e-7, guess="sad")
            eng.set_precision(0.0)
            mixed["scf"] = {"solves_per_s": round(1.0 / r3["seconds"], 4), "iterations": r3["niter"],
                            "E": r3["E"], "abs_dE_vs_fp64": abs(r3["E"] - g2["E"]),
                            "converged": bool(r3["converged"])}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        rate, sdesc, threads, t, stride = cpu_oracle_sample(basis, D_host, args.cpu_seconds)
        cpu = {"value": rate, "unit": "builds/s", "cores": threads, "kind": "port", "sample": sdesc}

    if rank == 0:
        line = {
            "metric": "Fock builds/s (FP64 closed-shell G(D))", "value": value, "unit": "builds/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "p50_ms": float(np.percentile(step_ms, 50)), "p99_ms": float(np.percentile(step_ms, 99)),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": desc, "nbasis": n, "integral_cutoff": INTEGRAL_CUTOFF, "prim_limit": PRIM_LIMIT,
                       "density": "core-Hamiltonian guess", "l2": "flushed between steps (256 MiB write)",
                       "parallelism": f"replicas x{world}"},
            "roofline": {"bound": "fp64", "kernel": f"fock_class_kernel<{','.join(str(x) for x in cls[4*top:4*top+4])}> ({tag})",
                         "achieved": round(top_tf, 4), "peak": round(peak_tf, 4), "unit": "TFLOP/s",
                         "frac": round(top_tf / peak_tf, 4) if peak_tf > 0 else None, "traffic": traffic,
                         "peak_source": "measured in-run: FP64 FMA probe kernel (qk_fp64_peak); "
                                        "MEASURED_PEAKS.json has no FP64 figure",
                         "all_classes_tflops": round(all_tf, 4),
                         "timing": "dominant class kernel timed alone with CUDA events, mean of "
                                   f"{nprof} builds; all_classes_tflops uses the concurrent build time"},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "builds/s", "h2d_bytes_per_step": 16 * n * n,
                    "d2h_bytes_per_step": 8 * n * n},
            "gpu_launches": int(launches) * args.steps,
            "clocks": clk,
            "scf": scf,
            "mixed": mixed,
            "bit_identical_host_vs_device": bit_identical,
            "classes": per_class,
            "autotune": None if tune_report is None else {
                "ms_default": round(tune_report["ms_default"], 4), "ms_tuned": round(tune_report["ms_tuned"], 4),
                "best_streams": tune_report["best_streams"],
                "streams_ms": {str(k): round(v, 4) for k, v in tune_report["streams"].items()},
                "warps_per_block": tune_report["warps"]},
        }
        print(json.dumps(line), flush=True)
    eng.close()
    if pg:
        pg.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="w32-631gs")
    ap.add_argument("--no-scf", action="store_true")
    ap.add_argument("--fp32-bound", type=float, default=1e-5,
                    help="mixed form: FP32 below this Schwarz bound product (0 = skip)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="default launch shapes (no autotuning)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--ref-step-seconds", type=float, default=6.0)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
