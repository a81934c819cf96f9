"""Generator of the per-class ERI device code (run at build time).

For every shell-quartet class (La Lb | Lc Ld) with La >= Lb, Lc >= Ld and
La+Lb >= Lc+Ld this script writes straight-line CUDA for

* the Head-Gordon--Pople vertical recursion (HGP eq. 6 and its ket analogue)
  from F_m(T) to the contracted intermediates [e0|f0], e = La..La+Lb,
  f = Lc..Lc+Ld (the same recursion QUICK's generated ``iclass_*`` blocks
  evaluate, ``src/gpu/gpu_eri_assembler_*.h``, ``src/subs/hrr.f90:1051-3456``);
* the horizontal recursion (a, b+1_i| = (a+1_i, b| + (A-B)_i (a, b| on the bra
  and the ket (``src/subs/hrr.f90:7-857``);
* the closed-shell J/K digestion of every integral with QUICK's Cartesian
  normalisation factors ``cons`` folded in.

Cartesian components follow QUICK's order (``src/basis.f90:589-720``): for a
total momentum L, z-exponent n ascending, then y-exponent m ascending.

Output: ``generated/eri_classes.cuh`` next to this file.
"""
from __future__ import annotations

import itertools
import math
import os
import sys

LMAX = 3  # f shells


def carts(L):
    out = []
    for n in range(L + 1):
        for m in range(L + 1 - n):
            out.append((L - n - m, m, n))
    return out


def ncart(L):
    return (L + 1) * (L + 2) // 2


def cons_of(c):
    """QUICK normalisation factor of a Cartesian component (src/basis.f90:589-720)."""
    L = sum(c)
    if L <= 1:
        return 1.0
    nz = sorted([x for x in c if x > 0], reverse=True)
    if L == 2:
        return 1.0 if nz == [2] else math.sqrt(3.0)
    if L == 3:
        if nz == [3]:
            return 1.0
        if nz == [2, 1]:
            return math.sqrt(5.0)
        return math.sqrt(5.0) * math.sqrt(3.0)
    raise ValueError(L)


def sub(v, i, k=1):
    w = list(v)
    w[i] -= k
    return tuple(w)


def add(v, i, k=1):
    w = list(v)
    w[i] += k
    return tuple(w)


ZERO = (0, 0, 0)
AX = "xyz"


class VRRGen:
    """Builds the VRR DAG for one class and emits code."""

    def __init__(self, Lab, Lcd, e_list, f_list, axis_order):
        self.Lab, self.Lcd = Lab, Lcd
        self.order = axis_order
        self.nodes = {}       # key -> (name, expr)
        self.emitted = []
        self.counter = 0
        self.e_list, self.f_list = e_list, f_list
        self.struct = []      # (name, key, record) in creation (topological) order
        self._last = None

    def pick(self, v):
        for i in self.order:
            if v[i] > 0:
                return i
        raise ValueError

    def name(self, e, f, m):
        key = (e, f, m)
        if key in self.nodes:
            return self.nodes[key]
        if min(e) < 0 or min(f) < 0:
            return None
        if e == ZERO and f == ZERO:
            nm = f"F{m}"
            self.nodes[key] = nm
            return nm
        terms = []
        # structural record: (kind, axis, a, b, c, d, g, n2, na) with operand names or None
        if f != ZERO:
            i = self.pick(f)
            f1 = sub(f, i)
            a = self.name(e, f1, m)
            b = self.name(e, f1, m + 1)
            c = d = g = None
            n2 = na = 0.0
            terms.append(f"QC{AX[i]} * {a}")
            terms.append(f"WQ{AX[i]} * {b}")
            if f1[i] > 0:
                f2 = sub(f1, i)
                c = self.name(e, f2, m)
                d = self.name(e, f2, m + 1)
                n2 = float(f1[i])
                terms.append(f"{float(f1[i])!r} * oo2e * ({c} - rho_e * {d})")
            if e[i] > 0:
                em = sub(e, i)
                g = self.name(em, f1, m + 1)
                na = float(e[i])
                terms.append(f"{float(e[i])!r} * oo2ze * {g}")
            rec = (1, i, a, b, c, d, g, n2, na)
        else:
            i = self.pick(e)
            e1 = sub(e, i)
            a = self.name(e1, ZERO, m)
            b = self.name(e1, ZERO, m + 1)
            c = d = None
            n2 = 0.0
            terms.append(f"PA{AX[i]} * {a}")
            terms.append(f"WP{AX[i]} * {b}")
            if e1[i] > 0:
                e2 = sub(e1, i)
                c = self.name(e2, ZERO, m)
                d = self.name(e2, ZERO, m + 1)
                n2 = float(e1[i])
                terms.append(f"{float(e1[i])!r} * oo2z * ({c} - rho_z * {d})")
            rec = (0, i, a, b, c, d, None, n2, 0.0)
        self._last = rec
        nm = f"v{self.counter}"
        self.counter += 1
        self.emitted.append(f"const double {nm} = " + " + ".join(terms) + ";")
        self.nodes[key] = nm
        self.struct.append((nm, key, self._last))
        return nm

    def build(self):
        targets = []
        for fi, f in enumerate(self.f_list):
            for ei, e in enumerate(self.e_list):
                targets.append((fi * len(self.e_list) + ei, self.name(e, f, 0)))
        return targets


def best_vrr(Lab, Lcd, e_list, f_list):
    best = None
    for order in itertools.permutations(range(3)):
        g = VRRGen(Lab, Lcd, e_list, f_list, order)
        t = g.build()
        if best is None or g.counter < best[0].counter:
            best = (g, t)
    return best


def hrr_plan(La, Lb, order=(0, 1, 2)):
    """Straight-line bra HRR: returns (lines, outputs) where the input column is
    ``src[idx(e)]`` for e in cart(La..La+Lb) and outputs (a,b) -> expression."""
    e_list = [c for L in range(La, La + Lb + 1) for c in carts(L)]
    e_index = {c: k for k, c in enumerate(e_list)}
    memo = {}
    lines = []
    cnt = [0]

    def node(a, b):
        if (a, b) in memo:
            return memo[(a, b)]
        if b == ZERO:
            nm = f"SRC({e_index[a]})"
            memo[(a, b)] = nm
            return nm
        i = next(k for k in order if b[k] > 0)
        b1 = sub(b, i)
        x = node(add(a, i), b1)
        y = node(a, b1)
        nm = f"h{cnt[0]}"
        cnt[0] += 1
        lines.append(f"const double {nm} = {x} + AB{AX[i]} * {y};")
        memo[(a, b)] = nm
        return nm

    outs = []
    for a in carts(La):
        for b in carts(Lb):
            outs.append(node(a, b))
    return lines, outs, len(e_list)


def best_hrr(La, Lb):
    best = None
    for order in itertools.permutations(range(3)):
        r = hrr_plan(La, Lb, order)
        if best is None or len(r[0]) < len(best[0]):
            best = r
    return best


COOP_MIN = 150   # NE*NF at or above which a class uses the warp-cooperative kernel
# f classes evaluated per lane although the f rule in is_coop would make them
# cooperative: their per-lane kernels keep almost all of their state in registers
# (0.1-5 KB local frames under -Xptxas -v) and ran 1.4-5.6x faster than the
# cooperative kernel on B200 (per-class CUDA-event times, 12 H2O / cc-pVTZ).  The
# other classes above the rules were measured per lane too and spill 15-27 KB per
# lane (dpdp, ddpp, ddds, ddfs, fppp, fpfs, fdds): 3-6x slower than cooperative.
PER_LANE = {(3, 0, 1, 1), (3, 0, 2, 0), (3, 0, 2, 1), (3, 0, 3, 0), (3, 1, 1, 0), (3, 1, 2, 0),
            (3, 2, 1, 0), (3, 3, 0, 0), (3, 3, 1, 0)}
SMEM_MAX = 227 * 1024   # shared memory of one block


def is_coop(La, Lb, Lc, Ld):
    """Warp-cooperative (one quartet per warp) or per-lane straight-line kernel."""
    Lab, Lcd = La + Lb, Lc + Ld
    NE = sum(ncart(L) for L in range(La, Lab + 1))
    NF = sum(ncart(L) for L in range(Lc, Lcd + 1))
    nint = ncart(La) * ncart(Lb) * ncart(Lc) * ncart(Ld)
    if (La, Lb, Lc, Ld) in PER_LANE:
        return False
    if max(La, Lb, Lc, Ld) >= 3:
        return NE * NF >= 60 or nint > 60
    return NE * NF >= COOP_MIN


def vrr_table(g, targets, M):
    """Level-ordered node table for the warp-cooperative VRR.

    Slot layout of the per-warp value array V: 0..M = scaled F_m, M+1 = 0.0,
    M+2+k = node k in level order.  Returns (rows, level_offsets, target_slots)."""
    level = {f"F{m}": 0 for m in range(M + 1)}
    for nm, key, rec in g.struct:
        ops = [x for x in rec[2:7] if x is not None]
        level[nm] = 1 + max(level[x] for x in ops)
    order = sorted(g.struct, key=lambda t: (level[t[0]], int(t[0][1:])))
    slot = {f"F{m}": m for m in range(M + 1)}
    for k, (nm, _, _) in enumerate(order):
        slot[nm] = M + 2 + k
    zero = M + 1
    rows = []
    for nm, key, rec in order:
        kind, axis, a, b, c, d, gg, n2, na = rec
        sl = lambda x: slot[x] if x is not None else zero  # noqa: E731
        rows.append((kind, axis, sl(a), sl(b), sl(c), sl(d), sl(gg), n2, na))
    nlev = max(level.values())
    off = [0]
    for L in range(1, nlev + 1):
        off.append(off[-1] + sum(1 for t in order if level[t[0]] == L))
    tslots = [slot[nm] for _, nm in sorted(targets)]
    return rows, off, tslots


def class_list(lmax=LMAX):
    pcls = [(a, b) for a in range(lmax + 1) for b in range(a + 1)]
    out = []
    for (La, Lb) in pcls:
        for (Lc, Ld) in pcls:
            if (La + Lb, La, Lb) < (Lc + Ld, Lc, Ld):
                continue
            out.append((La, Lb, Lc, Ld))
    return out


# Register ceiling of each per-lane class kernel (__maxnreg__).  ptxas's own choice
# for these kernels varies from build to build (psss got 80 registers in one build
# and 103 in another, dpss 128 and 170) and the higher counts cost occupancy; the
# ceilings below are the fastest of a sweep (no ceiling, 128, 85, 64 and the
# allocations ptxas chose) measured on 32 H2O / 6-31G*, per class kernel timed
# alone; for the per-lane f classes a 168 ceiling measured on 12 H2O / cc-pVTZ
# helped fpss (-19%) and slowed the others by 35-50%.  Classes not listed keep
# ptxas's choice (255 = no ceiling).
LANE_REGS = {(0, 0, 0, 0): 64, (1, 0, 0, 0): 80, (2, 0, 0, 0): 96, (2, 1, 0, 0): 128, (2, 2, 0, 0): 128,
             (1, 1, 1, 0): 128, (2, 0, 1, 0): 128, (3, 1, 0, 0): 168}


def emit_class(La, Lb, Lc, Ld):
    Lab, Lcd = La + Lb, Lc + Ld
    M = Lab + Lcd
    e_list = [c for L in range(La, Lab + 1) for c in carts(L)]
    f_list = [c for L in range(Lc, Lcd + 1) for c in carts(L)]
    NE, NF = len(e_list), len(f_list)
    na, nb, nc, nd = ncart(La), ncart(Lb), ncart(Lc), ncart(Ld)
    g, targets = best_vrr(Lab, Lcd, e_list, f_list)
    hb_lines, hb_outs, _ = best_hrr(La, Lb)
    hk_lines, hk_outs, _ = best_hrr(Lc, Ld)
    tag = f"{La}{Lb}{Lc}{Ld}"
    o = []
    o.append(f"// ---- class ({'spdf'[La]}{'spdf'[Lb]}|{'spdf'[Lc]}{'spdf'[Ld]}): "
             f"VRR nodes {g.counter}, bra HRR {len(hb_lines)}, ket HRR {len(hk_lines)}")
    o.append(f"template <> struct EriClass<{La}, {Lb}, {Lc}, {Ld}> {{")
    o.append(f"  static constexpr int M = {M}, NE = {NE}, NF = {NF};")
    o.append(f"  static constexpr int NA = {na}, NB = {nb}, NC = {nc}, ND = {nd};")
    o.append(f"  static constexpr int VRR_NODES = {g.counter}, HRR_BRA = {len(hb_lines)}, HRR_KET = {len(hk_lines)};")
    pf, qf = class_flops(La, Lb, Lc, Ld)
    o.append(f"  static constexpr double PRIM_FLOPS = {pf}.0, QUARTET_FLOPS = {qf}.0;")
    coop = is_coop(La, Lb, Lc, Ld)
    # VRR: accumulate acc[f*NE+e] += [e0|f0]^(0) with base F_m already scaled
    # (per-lane classes only; cooperative classes evaluate the node table instead)
    vrr_lines = []
    o_main = o
    o = vrr_lines
    o.append("  template <typename R>")
    o.append("  static __device__ __forceinline__ void vrr(const R* __restrict__ Fm, const VrrGeom<R>& G, R* __restrict__ acc) {")
    o.append("    const R PAx = G.PA[0], PAy = G.PA[1], PAz = G.PA[2];")
    o.append("    const R WPx = G.WP[0], WPy = G.WP[1], WPz = G.WP[2];")
    o.append("    const R QCx = G.QC[0], QCy = G.QC[1], QCz = G.QC[2];")
    o.append("    const R WQx = G.WQ[0], WQy = G.WQ[1], WQz = G.WQ[2];")
    o.append("    const R oo2z = G.oo2z, oo2e = G.oo2e, oo2ze = G.oo2ze, rho_z = G.rho_z, rho_e = G.rho_e;")
    o.append("    (void)PAx; (void)PAy; (void)PAz; (void)WPx; (void)WPy; (void)WPz;")
    o.append("    (void)QCx; (void)QCy; (void)QCz; (void)WQx; (void)WQy; (void)WQz;")
    o.append("    (void)oo2z; (void)oo2e; (void)oo2ze; (void)rho_z; (void)rho_e;")
    for m in range(M + 1):
        o.append(f"    const R F{m} = Fm[{m}];")
    for ln in g.emitted:
        o.append("    " + ln.replace("const double", "const R"))
    for idx, nm in targets:
        o.append(f"    acc[{idx}] += {nm};")
    o.append("  }")
    o = o_main
    if not coop:
        o.extend(vrr_lines)
    # bra HRR on one column: SRC(k) = src[k], out[a*NB+b]
    o.append("  static __device__ __forceinline__ void hrr_bra(const double* __restrict__ src, double* __restrict__ out, double ABx, double ABy, double ABz) {")
    o.append("    (void)ABx; (void)ABy; (void)ABz;")
    o.append("#define SRC(k) src[k]")
    for ln in hb_lines:
        o.append("    " + ln)
    for k, nm in enumerate(hb_outs):
        o.append(f"    out[{k}] = {nm};")
    o.append("#undef SRC")
    o.append("  }")
    # ket HRR on one (ab) row: SRC(k) = src[k*stride]
    o.append("  static __device__ __forceinline__ void hrr_ket(const double* __restrict__ src, int stride, double* __restrict__ out, double ABx, double ABy, double ABz) {")
    o.append("    (void)ABx; (void)ABy; (void)ABz;")
    o.append("#define SRC(k) src[(k) * stride]")
    for ln in hk_lines:
        o.append("    " + ln)
    for k, nm in enumerate(hk_outs):
        o.append(f"    out[{k}] = {nm};")
    o.append("#undef SRC")
    o.append("  }")
    # cons tables
    ca = ", ".join(repr(cons_of(c)) for c in carts(La))
    cb = ", ".join(repr(cons_of(c)) for c in carts(Lb))
    cc = ", ".join(repr(cons_of(c)) for c in carts(Lc))
    cd = ", ".join(repr(cons_of(c)) for c in carts(Ld))
    o.append(f"  static __device__ __forceinline__ double cons_a(int i) {{ const double t[{na}] = {{{ca}}}; return t[i]; }}")
    o.append(f"  static __device__ __forceinline__ double cons_b(int i) {{ const double t[{nb}] = {{{cb}}}; return t[i]; }}")
    o.append(f"  static __device__ __forceinline__ double cons_c(int i) {{ const double t[{nc}] = {{{cc}}}; return t[i]; }}")
    o.append(f"  static __device__ __forceinline__ double cons_d(int i) {{ const double t[{nd}] = {{{cd}}}; return t[i]; }}")
    o.append(f"  static constexpr bool COOP = {'true' if coop else 'false'};")
    o.append(f"  static constexpr int LANE_REGS = {LANE_REGS.get((La, Lb, Lc, Ld), 255)};")
    if coop:
        rows, off, tslots = vrr_table(g, targets, M)
        o.append(f"  static constexpr int NNODE = {len(rows)}, NLEVEL = {len(off) - 1}, NSLOT = {M + 2 + len(rows)};")
        o.append(f"  static __device__ const short* targets() {{ return vrr_targets_{tag}; }}")
        # packed node words: x = a | b << 16, y = c | d << 16, z = g | gidx << 16,
        # w = n2 | na << 8 (gidx = kind * 3 + axis; all small non-negative integers)
        words = []
        for (k, a, x, y, z, w, v, n2, na) in rows:
            assert max(x, y, z, w, v) < 65536 and float(n2).is_integer() and float(na).is_integer()
            words.append(f"{{{x} | ({y} << 16), {z} | ({w} << 16), {v} | ({k * 3 + a} << 16), "
                         f"{int(n2)} | ({int(na)} << 8)}}")
        pre = [f"__device__ const int4 vrr_ops_{tag}[{len(rows)}] = {{\n  " + ",\n  ".join(words) + "\n};",
               f"__device__ const short vrr_targets_{tag}[{len(tslots)}] = {{{', '.join(map(str, tslots))}}};"]
        # the levels as straight-line rounds of 32 nodes (a level's rounds are
        # independent, so their loads can be issued together)
        o.append("  static __device__ __forceinline__ void vrr_coop(double* __restrict__ V, const double* __restrict__ gs, int lane) {")
        o.append(f"    const int4* __restrict__ ops = vrr_ops_{tag};")
        for L in range(len(off) - 1):
            k0, k1 = off[L], off[L + 1]
            for r0 in range(k0, k1, 32):
                cnt = min(32, k1 - r0)
                guard = "" if cnt == 32 else f"if (lane < {cnt}) "
                o.append(f"    {guard}coop_node(V, gs, ops, {r0} + lane, {M + 2});")
            o.append("    __syncwarp();")
        o.append("  }")
        o = o[:1] + pre + o[1:]
    o.append("};")
    stats = dict(cls=tag, vrr=g.counter, hb=len(hb_lines), hk=len(hk_lines), NE=NE, NF=NF, coop=coop)
    return "\n".join(o), stats


def count_flops(expr_lines):
    """FP operations in emitted expressions: every binary * + - counts 1."""
    n = 0
    for ln in expr_lines:
        rhs = ln.split("=", 1)[1]
        n += rhs.count("*") + rhs.count(" + ") + rhs.count(" - ")
    return n


def boys_flops(M):
    # 7-term Taylor (7 mul + 6 fma = 19) plus, for M > 0, exp (1) and 3 per downward step;
    # scaling by the prefactor 1 per m
    return 19 + (1 + 3 * M if M > 0 else 0) + (M + 1)


def class_flops(La, Lb, Lc, Ld):
    """Algorithmic FP64 operation counts of one class: per primitive quartet and per
    contracted quartet (the model the benchmark's roofline uses)."""
    Lab, Lcd = La + Lb, Lc + Ld
    e_list = [c for L in range(La, Lab + 1) for c in carts(L)]
    f_list = [c for L in range(Lc, Lcd + 1) for c in carts(L)]
    g, _ = best_vrr(Lab, Lcd, e_list, f_list)
    hb, _, _ = best_hrr(La, Lb)
    hk, _, _ = best_hrr(Lc, Ld)
    NE, NF = len(e_list), len(f_list)
    na, nb, nc, nd = ncart(La), ncart(Lb), ncart(Lc), ncart(Ld)
    geom = 30   # zeta+eta, 1/(zeta+eta), rho, PQ, T, prefactor (div, sqrt counted 1 each), W-P, W-Q
    prim = geom + boys_flops(Lab + Lcd) + count_flops(g.emitted) + NE * NF
    quartet = NF * 2 * len(hb) + na * nb * 2 * len(hk) + na * nb * nc * nd * 13
    return prim, quartet


def main(out_dir, lmax=LMAX):
    os.makedirs(out_dir, exist_ok=True)
    parts = ["// Generated by gen_eri.py -- do not edit.",
             "#pragma once",
             "// one VRR node: kind 0 = bra step (PA, WP, oo2z, rho_z), 1 = ket step (QC, WQ, oo2e, rho_e)",
             "// One node of the cooperative VRR: V[base + k] from five slots of V and the",
             "// warp's geometry table gs (0-2 PA, 3-5 QC, 6-8 WP, 9-11 WQ, 12 1/2zeta,",
             "// 13 1/2eta, 14 rho/zeta, 15 rho/eta, 16 1/2(zeta+eta)); one formula for",
             "// bra (gidx 0-2) and ket (gidx 3-5) steps, unused operands on the zero slot.",
             "__device__ __forceinline__ void coop_node(double* __restrict__ V, const double* __restrict__ gs,",
             "                                          const int4* __restrict__ ops, int k, int base) {",
             "  const int4 w = __ldg(ops + k);",
             "  const int a = w.x & 0xffff, b = w.x >> 16, c = w.y & 0xffff, d = w.y >> 16;",
             "  const int g = w.z & 0xffff, gi = w.z >> 16, kind = gi >= 3 ? 1 : 0;",
             "  const double n2 = (double)(w.w & 0xff), na = (double)(w.w >> 8);",
             "  const double t = n2 * gs[12 + kind] * (V[c] - gs[14 + kind] * V[d]) + na * gs[16] * V[g];",
             "  V[base + k] = gs[gi] * V[a] + gs[6 + gi] * V[b] + t;",
             "}",
             "template <int La, int Lb, int Lc, int Ld> struct EriClass;"]
    stats = []
    for cls in class_list(lmax):
        txt, st = emit_class(*cls)
        parts.append(txt)
        stats.append(st)
    # pair classes (for the Schwarz kernels) and the class list for the host
    pcls = [(a, b) for a in range(lmax + 1) for b in range(a + 1)]
    parts.append("#define QK_PAIR_CLASS_LIST(X) " + " ".join(f"X({a}, {b})" for a, b in pcls))
    parts.append("#define QK_ERI_CLASS_LIST(X) \\")
    lines = [f"  X({a}, {b}, {c}, {d})" for (a, b, c, d) in class_list(lmax)]
    parts.append(" \\\n".join(lines))
    path = os.path.join(out_dir, "eri_classes.cuh")
    new = "\n".join(parts) + "\n"
    old = open(path).read() if os.path.exists(path) else None
    if new != old:
        with open(path, "w") as f:
            f.write(new)
    return stats


if __name__ == "__main__":
    out = sys.argv[1] if len(sys.argv) > 1 else os.path.join(os.path.dirname(os.path.abspath(__file__)), "generated")
    lmax = int(sys.argv[2]) if len(sys.argv) > 2 else LMAX
    for s in main(out, lmax):
        print(s)
