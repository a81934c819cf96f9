#!/usr/bin/env python
"""Freeze the reference-derived work model of the Fock build: per integral class,
the floating-point operations QUICK's own code spends, counted mechanically from
its source text.  Writes ``roofline/flops_per_class.json`` beside this script.

    python roofline/count_reference_flops.py <QUICK source tree>

Counting rules (each one names the reference text it reads):

* ``vrr`` -- the binary ``*``, ``+``, ``-`` and ``/`` operators in the generated
  vertical-recursion blocks ``src/gpu/iclass/iclass_<e>s<f>s.h`` that QUICK's
  ``ERint_vertical_*`` executes for the class.  Block selection evaluates the
  nested ``if`` conditions of ``src/gpu/gpu_eri_assembler_spd.h`` (all blocks
  up to [gs|gs]) for (I, J, K, L) = (La, Lb, Lc, Ld), plus, for blocks beyond
  [gs|gs], those of ``gpu_eri_assembler_spdf_1..8.h`` whose conditions hold
  (the accumulating versions; the ``_2`` copies are not counted).
* ``n_store`` -- the ``LOCSTORE(...) STORE_OPERATOR`` statements of those blocks:
  one contracted [e0|f0] element each, costed 2 (the contraction FMA).
* ``boys`` -- ``src/gpu/gpu_fmt.h:5-72`` for F_0..F_M, M = La+Lb+Lc+Ld, counted
  at its X > 33 branch (1/X, exp, sqrt(pi/4 * 1/X): 4 operations), the upward
  recursion (6 per m) and the scaling of every F_m by the primitive prefactor
  (``VY *= X2``, src/gpu/gpu_get2e_subs.h:269-271: 1 per m).  X > 33 is the
  cheapest branch, so this is a lower bound.
* ``hrr`` -- per basis-function quartet, the general case of ``hrrwhole``
  (``src/subs/hrr.f90:262-280``): Y = sum_i sum_j cL_i cR_j store(...) over the
  nL = prod_k (b_k + 1) bra and nR = prod_k (d_k + 1) ket terms of ``lefthrr``
  (3 operations per term pair), one multiply per extra coefficient, and the four
  ``cons`` factors.
* ``digest`` -- per basis-function quartet, the operators of the general
  closed-shell digestion block ``src/modules/include/eri.fh`` (the eight
  ``quick_qm_struct%o`` updates after ``DENSELK=...``), counted from the text.

Per class: ``prim`` = boys + vrr + 2 n_store (per primitive quartet),
``quartet`` = (hrr + digest) summed over the class's basis-function quartets
(per contracted shell quartet).  The Fock build's work is then
W = sum_class (prim x primitive quartets evaluated + quartet x quartets evaluated),
on the quartets that survive the CPU get2e's screens.
"""
from __future__ import annotations

import json
import os
import re
import sys

LETTERS = "spdfghik"
HERE = os.path.dirname(os.path.abspath(__file__))


def ncart(L):
    return (L + 1) * (L + 2) // 2


def cart(L):
    """QUICK's Cartesian order of a shell (src/basis.f90:589-720)."""
    out = []
    for nz in range(L + 1):
        for ny in range(L + 1 - nz):
            out.append((L - nz - ny, ny, nz))
    return out


# numeric literals, C (1.0E-01) and Fortran (2.d0, .5d0) forms, exponent signs included
_NUM = re.compile(r"(?<![A-Za-z_\d])(?:\d+\.\d*|\.\d+|\d+)(?:[eEdD][+-]?\d+)?")


def count_ops(expr: str) -> int:
    """Binary arithmetic operators of a C expression (unary signs excluded)."""
    e = _NUM.sub("0", expr)
    e = re.sub(r"\s+", "", e)
    n = 0
    for i, ch in enumerate(e):
        if ch in "*/":
            n += 1
        elif ch in "+-":
            prev = e[i - 1] if i > 0 else "("
            if prev.isalnum() or prev in "_)]":
                n += 1
    return n


def block_counts(path: str):
    """(operators, stores) of one generated VRR block."""
    src = open(path).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    src = re.sub(r"//[^\n]*", "", src)
    ops = stores = 0
    for stmt in src.split(";"):
        stmt = stmt.strip().strip("{}").strip()
        if not stmt:
            continue
        if "STORE_OPERATOR" in stmt:
            stores += 1
            ops += count_ops(stmt.split("STORE_OPERATOR", 1)[1])
        elif "=" in stmt:
            ops += count_ops(stmt.split("=", 1)[1])
    return ops, stores


def selected_blocks(assembler: str, I: int, J: int, K: int, L: int):
    """The iclass blocks an ERint_vertical_* assembler executes for (I, J, K, L):
    its nested if conditions evaluated, its #include lines collected."""
    src = open(assembler).read()
    body = src[src.index("{", src.index("ERint_vertical")) + 1:]
    stack = [True]          # truth of the enclosing blocks
    pending = None
    out = []
    i = 0
    env = {"I": I, "J": J, "K": K, "L": L}
    while i < len(body):
        if body.startswith("#include", i):
            j = body.index("\n", i)
            name = re.search(r'"([^"]+)"', body[i:j]).group(1)
            if all(stack):
                out.append(name)
            i = j
        elif body.startswith("if", i) and not (body[i - 1].isalnum() or body[i - 1] == "_"):
            j = body.index("{", i)
            cond = body[i + 2:j].strip()
            cond = cond.replace("&&", " and ").replace("||", " or ")
            pending = bool(eval(cond, {}, env))
            stack.append(pending)
            i = j + 1
        elif body[i] == "{":
            stack.append(True)
            i += 1
        elif body[i] == "}":
            stack.pop()
            if len(stack) == 0:
                break
            i += 1
        else:
            i += 1
    return out


def class_list(max_l=3):
    """The integral classes of this library: La >= Lb, Lc >= Ld, (La, Lb) >= (Lc, Ld)."""
    pairs = [(a, b) for a in range(max_l + 1) for b in range(a + 1)]
    return [(a, b, c, d) for (a, b) in pairs for (c, d) in pairs if (c, d) <= (a, b)]


def main(ref):
    gdir = os.path.join(ref, "src", "gpu")
    icl = os.path.join(gdir, "iclass")
    cache = {}

    def blk(name):
        if name not in cache:
            cache[name] = block_counts(os.path.join(icl, name))
        return cache[name]

    # the digestion block of the closed-shell CPU get2e (eri.fh), counted from its text
    eri = open(os.path.join(ref, "src", "modules", "include", "eri.fh")).read()
    # the closed-shell block: DENSELK is the alpha density alone (the open-shell
    # block before it adds denseb)
    k = re.search(r"DENSELK=quick_qm_struct%dense\(LLL,KKK\)\s*\n", eri).start()
    blockt = eri[k:eri.index("#endif", k)]
    upd = [ln for ln in blockt.splitlines() if "quick_qm_struct%o(" in ln and "=" in ln]
    digest = sum(count_ops(ln.split("=", 1)[1]) for ln in upd)

    spd = os.path.join(gdir, "gpu_eri_assembler_spd.h")
    spdf = [os.path.join(gdir, f"gpu_eri_assembler_spdf_{z}.h") for z in range(1, 9)]
    out = {}
    for (a, b, c, d) in class_list():
        names = selected_blocks(spd, a, b, c, d)
        for f in spdf:
            names += [n for n in selected_blocks(f, a, b, c, d) if n not in names]
        vrr = sum(blk(n)[0] for n in names)
        nst = sum(blk(n)[1] for n in names)
        M = a + b + c + d
        boys = 4 + 6 * M + (M + 1)
        hrr = 0
        for bx in cart(b):
            nL = (bx[0] + 1) * (bx[1] + 1) * (bx[2] + 1)
            for dx in cart(d):
                nR = (dx[0] + 1) * (dx[1] + 1) * (dx[2] + 1)
                hrr += ncart(a) * ncart(c) * (3 * nL * nR + (nL - 1) + (nR - 1) + 4)
        nint = ncart(a) * ncart(b) * ncart(c) * ncart(d)
        tag = LETTERS[a] + LETTERS[b] + LETTERS[c] + LETTERS[d]
        out[tag] = {"La": a, "Lb": b, "Lc": c, "Ld": d, "M": M, "blocks": names, "vrr": vrr, "n_store": nst,
                    "boys": boys, "prim": boys + vrr + 2 * nst, "hrr": hrr, "digest": digest * nint,
                    "quartet": hrr + digest * nint, "integrals": nint}
    meta = {"source": "QUICK source tree, counted by roofline/count_reference_flops.py",
            "digest_per_integral": digest,
            "rules": "see the script's docstring"}
    path = os.path.join(HERE, "flops_per_class.json")
    with open(path, "w") as f:
        json.dump({"meta": meta, "classes": out}, f, indent=1, sort_keys=True)
    print(path)
    for t in ("ssss", "psss", "psps", "dsds", "dddd", "fsfs", "ffff"):
        if t in out:
            print(t, out[t]["vrr"], out[t]["n_store"], out[t]["prim"], out[t]["quartet"])


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: count_reference_flops.py <QUICK source tree>")
    main(sys.argv[1])
