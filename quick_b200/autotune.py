"""Autotuner for the Fock build's launch shapes and the mixed form's switch bound.

The Fock build runs one persistent kernel per integral class (blocks loop over
the class's work items), so its launch shape is free: any shape computes the
same integrals and, through the int64 accumulation, the same Fock matrix bit for
bit.  What the shape changes is speed -- occupancy against registers and shared
memory, and how the class kernels share the GPU.  The tuner measures, on the
caller's molecule and density, with CUDA events:

1. per class, the warps per block (``qk_set_class_launch``): every candidate is
   applied to all classes at once, the classes are timed one by one in the same
   builds (``qk_set_profiling`` events), and each class keeps its fastest shape;
2. the stream count (``qk_set_streams``): class kernels concurrent over 1, 2 or 4
   streams, or one after another -- whole builds timed;
3. the s/p classes as one merged kernel (``qk_set_merge_sp``) or one launch per
   class, with each stream count -- whole builds timed (the merged launch pays on
   small molecules, whose builds are launch-bound, and loses on large ones, where
   it runs every s/p class at the largest one's register allocation);
4. optionally (:func:`tune_precision`) the mixed form's Schwarz switch bound:
   the fastest bound whose SCF energy stays within ``tol`` of plain FP64.

The reference has no counterpart (its kernels are launched with fixed shapes,
``src/gpu/gpu_get2e.cu``); this module is the B200 build's own tuner.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._native import check, lib

SPDF = "spdf"


def _P(a):
    return ctypes.c_void_p(a.ctypes.data)


def classes(eng):
    """[(index, name, max warps per block)] of the compiled integral classes."""
    L = lib()
    n = 256
    cls = np.zeros(4 * n, dtype=np.int32)
    nc = L.qk_class_profile(ctypes.c_void_p(eng.h), n, _P(cls), None, None, None, None, None, None, None)
    out = []
    for i in range(nc):
        w, mw, b, g = (ctypes.c_int(0) for _ in range(4))
        check(L.qk_class_launch(ctypes.c_void_p(eng.h), i, ctypes.byref(w), ctypes.byref(mw), ctypes.byref(b),
                                ctypes.byref(g)), "qk_class_launch")
        out.append((i, "".join(SPDF[x] for x in cls[4 * i:4 * i + 4]), mw.value))
    return out


def class_times(eng, D, reps: int = 3):
    """Per-class kernel milliseconds (minimum over ``reps`` builds, classes timed
    one after another with CUDA events)."""
    import torch
    L = lib()
    n = 256
    ms = np.zeros(n, dtype=np.float32)
    best = None
    o = torch.zeros_like(D)
    check(L.qk_set_profiling(ctypes.c_void_p(eng.h), 1, 0), "qk_set_profiling")
    try:
        for _ in range(reps):
            o.zero_()
            eng.fock2e(D, o=o)
            nc = L.qk_class_profile(ctypes.c_void_p(eng.h), n, None, _P(ms), None, None, None, None, None, None)
            t = ms[:nc].astype(np.float64).copy()
            best = t if best is None else np.minimum(best, t)
    finally:
        L.qk_set_profiling(ctypes.c_void_p(eng.h), 0, 0)
    return best


def build_ms(eng, D, reps: int = 5):
    """Milliseconds per whole build (minimum over ``reps``, CUDA events)."""
    import torch
    o = torch.zeros_like(D)
    eng.fock2e(D, o=o)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = float("inf")
    for _ in range(reps):
        o.zero_()
        e0.record()
        eng.fock2e(D, o=o)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return best


def set_shape(eng, idx: int, warps: int, blocks_per_sm: int = 0):
    check(lib().qk_set_class_launch(ctypes.c_void_p(eng.h), idx, int(warps), int(blocks_per_sm)),
          "qk_set_class_launch")


def tune(eng, D, warps=(1, 2, 4, 8), streams=(0, 1, 2, 4), reps: int = 3):
    """Tune ``eng``'s launch shapes on density ``D`` (a CUDA float64 tensor) and
    leave the best ones applied.  Returns a report of every measurement."""
    eng.fock2e(D)                      # tables and work lists built before timing
    cls = classes(eng)
    ms_default = build_ms(eng, D, reps)
    per = {name: {} for _, name, _ in cls}
    for w in warps:
        for i, _, mw in cls:
            set_shape(eng, i, min(w, mw))
        t = class_times(eng, D, reps)
        for i, name, mw in cls:
            if t[i] > 0:
                per[name][min(w, mw)] = float(t[i])
    chosen = {}
    for i, name, mw in cls:
        if per[name]:
            w = min(per[name], key=per[name].get)
            chosen[name] = w
            set_shape(eng, i, w)
        else:
            set_shape(eng, i, 0)
    st = {}
    for merged in (False, True):
        eng.set_merge_sp(merged)
        for s in streams:
            eng.set_streams(s)
            st[(s, merged)] = build_ms(eng, D, reps)
    best_s, best_m = min(st, key=st.get)
    eng.set_streams(best_s)
    eng.set_merge_sp(best_m)
    return {"ms_default": ms_default, "ms_tuned": st[(best_s, best_m)],
            "streams": {s: t for (s, m), t in st.items() if not m},
            "streams_merged_sp": {s: t for (s, m), t in st.items() if m},
            "best_streams": best_s, "merge_sp": best_m, "warps": chosen, "class_ms": per}


def tune_precision(make_rhf, bounds=(1e-6, 1e-5, 1e-4), tol: float = 1e-6, denserms: float = 1e-7,
                   reps: int = 3):
    """Pick the mixed form's switch bound: for each bound, an SCF against the FP64
    one (``make_rhf()`` returns a fresh :class:`quick_b200.scf.RHF`) and the build
    time at its converged density; the fastest bound with |dE| <= tol wins
    (0.0 = plain FP64 when none qualifies)."""
    ref = make_rhf()
    r0 = ref.run(denserms=denserms)
    t0 = build_ms(ref.eng, r0["D"], reps)
    rows = {0.0: {"dE": 0.0, "build_ms": t0, "niter": r0["niter"]}}
    best, best_t = 0.0, t0
    for b in bounds:
        rhf = make_rhf()
        rhf.eng.set_precision(b)
        r = rhf.run(denserms=denserms)
        t = build_ms(rhf.eng, r0["D"], reps)
        dE = abs(r["E"] - r0["E"])
        rows[b] = {"dE": dE, "build_ms": t, "niter": r["niter"], "fp32_quartets": rhf.eng.fp32_quartets()}
        if dE <= tol and r["converged"] and t < best_t:
            best, best_t = b, t
    return {"best_bound": best, "E_fp64": r0["E"], "bounds": rows}
