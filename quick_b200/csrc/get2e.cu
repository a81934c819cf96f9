// B200-native closed-shell two-electron Fock build (QUICK "get2e").
//
// Replaces the reference path gpu_get_cshell_eri_ -> get2e -> get2e_kernel_*
// (src/gpu/gpu_get2e_getxc_drivers.h:24-123, src/gpu/cuda/gpu_get2e.cu:594-637,
// src/gpu/gpu_get2e_subs.h:664-1046) with:
//
//  * shell pairs split into s/p/d "Qshells" (SP shells give one s and one p),
//    bucketed by (La, Lb, contraction length) and sorted by Schwarz bound, so the
//    Schwarz test of a bra pair against a bucket is a prefix and every lane of a
//    warp runs the same primitive loop;
//  * one warp per work item = (bra pair, up to 32 consecutive ket pairs), one
//    lane per shell quartet, straight-line HGP VRR/HRR generated per class
//    (gen_eri.py), FP64 throughout;
//  * J/K digestion into a full int64 fixed-point accumulator A (scale 2^44):
//    J over the bra is warp-reduced before its atomics; G = A + A^T at the end.
//    Integer addition is exact and order independent, so the Fock matrix is
//    bit-identical from run to run.
//
// Screening follows QUICK's CPU path (src/modules/include/eri.fh:178-189, 274,
// 309-310): a quartet survives when Y_ij*Y_kl > integralCutoff and
// Y_ij*Y_kl*DNmax > integralCutoff, a primitive quartet when
// DNmax*cutprim_ij*cutprim_kl > primLimit.  Y, cutprim and the density screen
// are indexed by the reference's (unsplit) shells.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <tuple>
#include <vector>

#include <cub/device/device_scan.cuh>

#include "quick_b200.h"
#include "common.cuh"

namespace qk {

#include "generated/eri_classes.cuh"

// ------------------------------------------------------------------ device data
struct DevData {
    int nbasis, nshell;
    const double* __restrict__ xyz;      // 3*natom
    const int* __restrict__ q_atom;      // per Qshell
    const int* __restrict__ q_f0;
    const int* __restrict__ q_parent;
    const int* __restrict__ q_ltop;      // per Qshell: the top angular momentum of its shell (1 for SP)
    const int* __restrict__ pr_qa;       // per pair
    const int* __restrict__ pr_qb;
    const int* __restrict__ pr_pp0;
    const int* __restrict__ pr_npp;
    const int* __restrict__ pr_pps;      // stride between a pair's primitive pairs
    const double* __restrict__ pr_Y;
    // per pair, what the per-lane quartet code would otherwise reach through chains
    // of dependent loads (pair -> Qshell -> parent shell / atom -> coordinates):
    // (parent shell of a, of b, first function of a, of b); the top angular
    // momenta of the two shells summed; and (Ax, Ay), (Az, ABx), (ABy, ABz) with A
    // the centre of the first Qshell and AB = A - B
    const int4* __restrict__ pr_sh;
    const int* __restrict__ pr_lt;
    const double2* __restrict__ pr_geo;   // 3 per pair
    // per primitive pair, five 16-byte fields (one vector load each):
    // (zeta, 1/(2 zeta)), (K, cutprim), (Px, Py), (Pz, PAx), (PAy, PAz) with
    // K = exp(-ab/zeta R_AB^2)/zeta c_a c_b sqrt(X0) and PA = P - centre of the first shell
    const double2* __restrict__ pp_zo;
    const double2* __restrict__ pp_kc;
    const double2* __restrict__ pp_pxy;
    const double2* __restrict__ pp_pzax;
    const double2* __restrict__ pp_payz;
    const double* __restrict__ boys;     // kBoysNT x kBoysNM
    const double2* __restrict__ boys8;   // row tables, M = 0..4 kMaxL (boys_row_tables)
    const double* __restrict__ D;        // nbasis^2
    const double* __restrict__ cutmat;   // nshell^2
    unsigned long long* __restrict__ A;  // nbasis^2 fixed point
    unsigned long long* stats;           // optional: [quartets computed, primitive quartets computed]
    double cut, primLimit;
    int boys_mode;                       // qk_set_boys: 0 accurate; 1 QUICK CPU order; 2 QUICK GPU order
    int exchange_only;                   // 1: the K part alone (the spin-density half of a UHF build)
};

__device__ __forceinline__ void atomic_fixed(unsigned long long* addr, double v) {
    long long iv = __double2ll_rn(v * kFixedScale);
    atomicAdd(addr, (unsigned long long)iv);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Contracted [e0|f0] over the primitive pairs of a bra and a ket pair.
// acc[f*NE + e]; prim_screen applies QUICK's primitive cutoff.  R is the type of
// the vertical recursion and of acc: double for the plain path, float for the
// small-bound quartets of the mixed form.  Geometry and the Boys function are
// always evaluated in FP64 and rounded to R afterwards.
// mq: the order QUICK's CPU get2e evaluates the Boys function at for this quartet
// (the sum of the four shells' top angular momenta, SP shells counting 1), used by
// the QUICK-faithful mode 1 of qk_set_boys.
template <int La, int Lb, int Lc, int Ld, typename R = double>
__device__ __forceinline__ void contract_quartet(const DevData& d, const double2* __restrict__ bt, int bp0, int bnp,
                                                 int bps, int kp0, int knp, int kps,
                                                 const double C[3], double dnmax, bool prim_screen, int mq,
                                                 R* acc, int* nprim_done) {
    using Cls = EriClass<La, Lb, Lc, Ld>;
    constexpr int M = Cls::M;
#pragma unroll
    for (int i = 0; i < Cls::NE * Cls::NF; ++i) acc[i] = R(0);
    // ket primitive outer, bra primitive inner: the lane's own ket data is read
    // once per ket primitive; the inner loop reads only the bra data, which is
    // the same for the whole warp
    for (int j = 0; j < knp; ++j) {
        const int pj = kp0 + j * kps;
        const double2 kcj = __ldg(d.pp_kc + pj), zoj = __ldg(d.pp_zo + pj);
        const double2 qxy = __ldg(d.pp_pxy + pj), qzax = __ldg(d.pp_pzax + pj);
        const double cutj = kcj.y, eta = zoj.x, oo2e = zoj.y, Kcd = kcj.x;
        const double Qx = qxy.x, Qy = qxy.y, Qz = qzax.x;
        for (int i = 0; i < bnp; ++i) {
            const int pi = bp0 + i * bps;
            const double2 kci = __ldg(d.pp_kc + pi);
            const double cut1 = dnmax * kci.y;
            if (prim_screen && !(cut1 * cutj > d.primLimit)) continue;
            ++*nprim_done;
            const double2 zoi = __ldg(d.pp_zo + pi), pxy = __ldg(d.pp_pxy + pi);
            const double2 pzax = __ldg(d.pp_pzax + pi), payz = __ldg(d.pp_payz + pi);
            const double zeta = zoi.x, oo2z = zoi.y, Kab = kci.x;
            const double Px = pxy.x, Py = pxy.y, Pz = pzax.x;
            const double PAx = pzax.y, PAy = payz.x, PAz = payz.y;
            const double s = zeta + eta;
            const double rs = rsqrt(s);            // 1/sqrt(zeta+eta), 1 ulp
            const double inv_s = rs * rs;
            const double rho_z = eta * inv_s, rho_e = zeta * inv_s;
            const double rho = zeta * rho_z;
            const double PQx = Px - Qx, PQy = Py - Qy, PQz = Pz - Qz;
            const double T = rho * (PQx * PQx + PQy * PQy + PQz * PQz);
            const double pref = Kab * Kcd * rs;
            double F[M + 1];
            if (d.boys_mode)
                boys_quick_scaled<M>(T, pref, F, d.boys_mode == 1 ? mq : M);
            else
                boys_scaled_rows<M>(T, pref, bt, F);
            VrrGeom<R> G;
            G.PA[0] = R(PAx); G.PA[1] = R(PAy); G.PA[2] = R(PAz);
            G.WP[0] = R(-rho_z * PQx); G.WP[1] = R(-rho_z * PQy); G.WP[2] = R(-rho_z * PQz);
            G.QC[0] = R(Qx - C[0]); G.QC[1] = R(Qy - C[1]); G.QC[2] = R(Qz - C[2]);
            G.WQ[0] = R(rho_e * PQx); G.WQ[1] = R(rho_e * PQy); G.WQ[2] = R(rho_e * PQz);
            G.oo2z = R(oo2z);
            G.oo2e = R(oo2e);
            G.oo2ze = R(0.5 * inv_s);
            G.rho_z = R(rho_z);
            G.rho_e = R(rho_e);
            R Fr[M + 1];
#pragma unroll
            for (int m = 0; m <= M; ++m) Fr[m] = R(F[m]);
            Cls::template vrr<R>(Fr, G, acc);
        }
    }
}

// One quartet (bra pair P, ket pair Q): integrals, J/K digestion.
// Lane-private updates go straight to A; the bra J block is returned in jab
// (already weighted) for the warp reduction.
template <int La, int Lb, int Lc, int Ld, bool FP32>
__device__ __forceinline__ void fock_quartet(const DevData& d, const double2* __restrict__ bt, int P, int Q,
                                             double* jab_out, int* nq_done, int* np_done) {
    using Cls = EriClass<La, Lb, Lc, Ld>;
    constexpr int NA = Cls::NA, NB = Cls::NB, NC = Cls::NC, ND = Cls::ND;
    constexpr int NE = Cls::NE, NF = Cls::NF, NAB = NA * NB;
    const int n = d.nbasis, ns = d.nshell;
    const int4 shP = d.pr_sh[P], shQ = d.pr_sh[Q];
    const int sa = shP.x, sb = shP.y, sc = shQ.x, sd = shQ.y;
    const double* cm = d.cutmat;
    double dnmax = fmax(4.0 * cm[sa * ns + sb], 4.0 * cm[sc * ns + sd]);
    dnmax = fmax(dnmax, fmax(cm[sa * ns + sd], cm[sa * ns + sc]));
    dnmax = fmax(dnmax, fmax(cm[sb * ns + sc], cm[sb * ns + sd]));
    const double ct = d.pr_Y[P] * d.pr_Y[Q];
    // the CPU get2e's two tests (Y_P Y_Q > cut, then with DNmax): the work list may
    // have been built at a tighter cutoff than the one in force
    if (!(ct > d.cut) || !(ct * dnmax > d.cut)) return;
    ++*nq_done;

    const double2 gp1 = d.pr_geo[3 * P + 1], gp2 = d.pr_geo[3 * P + 2];
    const double2 gq0 = d.pr_geo[3 * Q], gq1 = d.pr_geo[3 * Q + 1], gq2 = d.pr_geo[3 * Q + 2];
    const double AB[3] = {gp1.y, gp2.x, gp2.y};
    const double Cc[3] = {gq0.x, gq0.y, gq1.x};
    const double CD[3] = {gq1.y, gq2.x, gq2.y};

    const int mq = d.pr_lt[P] + d.pr_lt[Q];
    double acc[NE * NF];
    if constexpr (FP32) {
        // mixed form: small-bound quartet, vertical recursion and contraction in FP32
        float accf[NE * NF];
        contract_quartet<La, Lb, Lc, Ld, float>(d, bt, d.pr_pp0[P], d.pr_npp[P], d.pr_pps[P], d.pr_pp0[Q],
                                                d.pr_npp[Q], d.pr_pps[Q], Cc, dnmax, true, mq, accf, np_done);
#pragma unroll
        for (int i = 0; i < NE * NF; ++i) acc[i] = (double)accf[i];
    } else {
        contract_quartet<La, Lb, Lc, Ld>(d, bt, d.pr_pp0[P], d.pr_npp[P], d.pr_pps[P], d.pr_pp0[Q], d.pr_npp[Q],
                                         d.pr_pps[Q], Cc, dnmax, true, mq, acc, np_done);
    }

    // bra HRR per ket column
    double t1[NF * NAB];
#pragma unroll
    for (int f = 0; f < NF; ++f) Cls::hrr_bra(acc + f * NE, t1 + f * NAB, AB[0], AB[1], AB[2]);

    const int fa = shP.z, fb = shP.w, fc = shQ.z, fd = shQ.w;
    // degeneracy of the unique quartet (pairs are unordered, bra/ket unordered);
    // a pair of two different Qshells starts at two different functions
    const double deg = (fa != fb ? 2.0 : 1.0) * (fc != fd ? 2.0 : 1.0) * (P != Q ? 2.0 : 1.0);
    const double wJ = d.exchange_only ? 0.0 : 0.25 * deg;   // 2 * deg/8
    const double wK = -0.0625 * deg;                        // -1/2 * deg/8

    double Dab[NAB], Dcd[NC * ND], Dbd[NB * ND], Dad[NA * ND], Dbc[NB * NC], Dac[NA * NC];
#pragma unroll
    for (int a = 0; a < NA; ++a)
#pragma unroll
        for (int b = 0; b < NB; ++b) Dab[a * NB + b] = d.D[(fa + a) * n + fb + b];
#pragma unroll
    for (int c = 0; c < NC; ++c)
#pragma unroll
        for (int e = 0; e < ND; ++e) Dcd[c * ND + e] = d.D[(fc + c) * n + fd + e];
#pragma unroll
    for (int b = 0; b < NB; ++b)
#pragma unroll
        for (int e = 0; e < ND; ++e) Dbd[b * ND + e] = d.D[(fb + b) * n + fd + e];
#pragma unroll
    for (int a = 0; a < NA; ++a)
#pragma unroll
        for (int e = 0; e < ND; ++e) Dad[a * ND + e] = d.D[(fa + a) * n + fd + e];
#pragma unroll
    for (int b = 0; b < NB; ++b)
#pragma unroll
        for (int c = 0; c < NC; ++c) Dbc[b * NC + c] = d.D[(fb + b) * n + fc + c];
#pragma unroll
    for (int a = 0; a < NA; ++a)
#pragma unroll
        for (int c = 0; c < NC; ++c) Dac[a * NC + c] = d.D[(fa + a) * n + fc + c];

    double jcd[NC * ND], kac[NA * NC], kbc[NB * NC], kad[NA * ND], kbd[NB * ND];
#pragma unroll
    for (int i = 0; i < NC * ND; ++i) jcd[i] = 0.0;
#pragma unroll
    for (int i = 0; i < NA * NC; ++i) kac[i] = 0.0;
#pragma unroll
    for (int i = 0; i < NB * NC; ++i) kbc[i] = 0.0;
#pragma unroll
    for (int i = 0; i < NA * ND; ++i) kad[i] = 0.0;
#pragma unroll
    for (int i = 0; i < NB * ND; ++i) kbd[i] = 0.0;

#pragma unroll
    for (int a = 0; a < NA; ++a) {
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const int ab = a * NB + b;
            double I[NC * ND];
            Cls::hrr_ket(t1 + ab, NAB, I, CD[0], CD[1], CD[2]);
            const double cab = Cls::cons_a(a) * Cls::cons_b(b);
            double jsum = 0.0;
#pragma unroll
            for (int c = 0; c < NC; ++c) {
#pragma unroll
                for (int e = 0; e < ND; ++e) {
                    const double v = I[c * ND + e] * (cab * Cls::cons_c(c) * Cls::cons_d(e));
                    jsum = fma(v, Dcd[c * ND + e], jsum);
                    jcd[c * ND + e] = fma(v, Dab[ab], jcd[c * ND + e]);
                    kac[a * NC + c] = fma(v, Dbd[b * ND + e], kac[a * NC + c]);
                    kbc[b * NC + c] = fma(v, Dad[a * ND + e], kbc[b * NC + c]);
                    kad[a * ND + e] = fma(v, Dbc[b * NC + c], kad[a * ND + e]);
                    kbd[b * ND + e] = fma(v, Dac[a * NC + c], kbd[b * ND + e]);
                }
            }
            jab_out[ab] = wJ * jsum;
        }
    }
    unsigned long long* A = d.A;
    if (!d.exchange_only) {
#pragma unroll
        for (int c = 0; c < NC; ++c)
#pragma unroll
            for (int e = 0; e < ND; ++e) atomic_fixed(A + (size_t)(fc + c) * n + fd + e, wJ * jcd[c * ND + e]);
    }
#pragma unroll
    for (int a = 0; a < NA; ++a)
#pragma unroll
        for (int c = 0; c < NC; ++c) atomic_fixed(A + (size_t)(fa + a) * n + fc + c, wK * kac[a * NC + c]);
#pragma unroll
    for (int b = 0; b < NB; ++b)
#pragma unroll
        for (int c = 0; c < NC; ++c) atomic_fixed(A + (size_t)(fb + b) * n + fc + c, wK * kbc[b * NC + c]);
#pragma unroll
    for (int a = 0; a < NA; ++a)
#pragma unroll
        for (int e = 0; e < ND; ++e) atomic_fixed(A + (size_t)(fa + a) * n + fd + e, wK * kad[a * ND + e]);
#pragma unroll
    for (int b = 0; b < NB; ++b)
#pragma unroll
        for (int e = 0; e < ND; ++e) atomic_fixed(A + (size_t)(fb + b) * n + fd + e, wK * kbd[b * ND + e]);
}

// ------------------------------------------------------------------ warp-cooperative classes
// High angular momentum classes (NE*NF >= 150) evaluate ONE quartet per warp:
// the VRR runs as a level-ordered node table over the 32 lanes with the values in
// shared memory, the bra HRR runs one ket column per lane, the ket HRR one bra
// row per lane, and the digestion one output element per lane (a fixed-order dot
// product, so results stay deterministic).

// F_m(T) for one m (lane-parallel Boys): Taylor on the grid, or upward recursion
// from the asymptotic F_0 above the grid.
__device__ __forceinline__ double boys_one(int m, double T, const double* __restrict__ tab) {
    if (T < kBoysTmax) {
        const int k = __double2int_rn(T * kBoysInvDT);
        const double u = k * kBoysDT - T;
        const double* t = tab + k * kBoysNM + m;
        double f = __ldg(t + 6) * (1.0 / 720.0);
        f = fma(f, u, __ldg(t + 5) * (1.0 / 120.0));
        f = fma(f, u, __ldg(t + 4) * (1.0 / 24.0));
        f = fma(f, u, __ldg(t + 3) * (1.0 / 6.0));
        f = fma(f, u, __ldg(t + 2) * 0.5);
        f = fma(f, u, __ldg(t + 1));
        return fma(f, u, __ldg(t + 0));
    }
    double f = kHalfSqrtPi * rsqrt(T);
    if (m > 0) {
        const double e = exp(-T), h = 0.5 / T;
        for (int j = 0; j < m; ++j) f = fma((double)(2 * j + 1), f, -e) * h;
    }
    return f;
}

template <int La, int Lb, int Lc, int Ld>
struct CoopLayout {
    using Cls = EriClass<La, Lb, Lc, Ld>;
    static constexpr int NAB = Cls::NA * Cls::NB, NCD = Cls::NC * Cls::ND;
    static constexpr int ACC = Cls::NE * Cls::NF;
    static constexpr int HRR = Cls::NF * NAB + NAB * NCD;
    static constexpr int WORK = Cls::NSLOT > HRR ? Cls::NSLOT : HRR;
    static constexpr int DBLK = NAB + NCD + Cls::NB * Cls::ND + Cls::NA * Cls::ND + Cls::NB * Cls::NC +
                                Cls::NA * Cls::NC;
    static constexpr int GEO = 24;                       // the VRR's geometry table (17 used)
    static constexpr int PER_WARP = ACC + WORK + DBLK + GEO;   // doubles
    // warps per block: as many as fit 227 KB of shared memory, at most 4
    static constexpr int FIT = (227 * 1024) / (8 * PER_WARP);
    static constexpr int WARPS = FIT < 1 ? 1 : (FIT > 4 ? 4 : FIT);
    static_assert(8 * PER_WARP <= 227 * 1024, "cooperative class does not fit in shared memory");
};

// Contracted [e0|f0] of one quartet into acc (shared, per warp), the VRR done
// level by level over the 32 lanes with its values in V (shared, per warp).
template <int La, int Lb, int Lc, int Ld>
__device__ __forceinline__ void coop_contract(const DevData& d, int bp0, int bnp, int bps, int kp0, int knp, int kps,
                                              double Cx, double Cy, double Cz, double dnmax, bool screen, int mq,
                                              double* acc, double* V, int lane, int* np_done) {
    using Cls = EriClass<La, Lb, Lc, Ld>;
    using Lay = CoopLayout<La, Lb, Lc, Ld>;
    constexpr int M = Cls::M;
    for (int t = lane; t < Lay::ACC; t += 32) acc[t] = 0.0;
    if (lane == 0) V[M + 1] = 0.0;
    const short* __restrict__ tgt = Cls::targets();
    double* gs = acc + Lay::PER_WARP - Lay::GEO;          // this warp's geometry table
    for (int i = 0; i < bnp; ++i) {
        const int pi = bp0 + i * bps;
        const double2 zoi = __ldg(d.pp_zo + pi), kci = __ldg(d.pp_kc + pi), pxy = __ldg(d.pp_pxy + pi);
        const double2 pzax = __ldg(d.pp_pzax + pi), payz = __ldg(d.pp_payz + pi);
        const double zeta = zoi.x, oo2z = zoi.y, Kab = kci.x;
        const double cut1 = dnmax * kci.y;
        const double Px = pxy.x, Py = pxy.y, Pz = pzax.x;
        const double PAx = pzax.y, PAy = payz.x, PAz = payz.y;
        for (int j = 0; j < knp; ++j) {
            const int pj = kp0 + j * kps;
            const double2 kcj = __ldg(d.pp_kc + pj);
            if (screen && !(cut1 * kcj.y > d.primLimit)) continue;   // warp-uniform
            if (lane == 0) ++*np_done;
            const double2 zoj = __ldg(d.pp_zo + pj), qxy = __ldg(d.pp_pxy + pj), qzax = __ldg(d.pp_pzax + pj);
            const double eta = zoj.x, oo2e = zoj.y;
            const double Qx = qxy.x, Qy = qxy.y, Qz = qzax.x;
            const double s = zeta + eta, rs = rsqrt(s), inv_s = rs * rs;
            const double rho_z = eta * inv_s, rho_e = zeta * inv_s, rho = zeta * rho_z;
            const double PQx = Px - Qx, PQy = Py - Qy, PQz = Pz - Qz;
            const double T = rho * (PQx * PQx + PQy * PQy + PQz * PQz);
            const double pref = Kab * kcj.x * rs;
            if (lane <= M)
                V[lane] = (d.boys_mode ? boys_quick_one(lane, d.boys_mode == 1 ? mq : M, T) : boys_one(lane, T, d.boys)) *
                          pref;
            if (lane == 0) {
                gs[0] = PAx; gs[1] = PAy; gs[2] = PAz;
                gs[3] = Qx - Cx; gs[4] = Qy - Cy; gs[5] = Qz - Cz;
                gs[6] = -rho_z * PQx; gs[7] = -rho_z * PQy; gs[8] = -rho_z * PQz;
                gs[9] = rho_e * PQx; gs[10] = rho_e * PQy; gs[11] = rho_e * PQz;
                gs[12] = oo2z; gs[13] = oo2e; gs[14] = rho_z; gs[15] = rho_e; gs[16] = 0.5 * inv_s;
            }
            __syncwarp();
            Cls::vrr_coop(V, gs, lane);
            for (int t = lane; t < Lay::ACC; t += 32) acc[t] += V[tgt[t]];
            __syncwarp();
        }
    }
}

// Asynchronous global -> shared copies (cp.async, 8 bytes), used to bring a
// quartet's density blocks in while its VRR runs.
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Digestion of one quartet by the warp, one group of outputs at a time (J_ab,
// J_cd, K_ac, K_bc, K_ad, K_bd).  A group has NOUT outputs, each a dot product
// over the terms (k1, k2), k1 < N1, k2 < N2, of the integral I[base(o) + k1*ST1 +
// k2*ST2] and the density element Dv[k1*N2 + k2].  S lanes share an output (S a
// power of two <= N1, fixed per group at compile time): each takes every S-th k1
// and all k2, and the partial sums meet in a fixed shuffle tree, so the sums do
// not depend on timing.  S minimises rounds x (terms per lane + shuffle steps +
// the round's address and atomic work):
// groups with few outputs and long sums (J_cd, K_ad, K_bd of the d classes) no
// longer run on a handful of lanes while the others wait.
__host__ __device__ constexpr int digest_cost(int nout, int n1, int n2, int s) {
    int lg = 0;
    for (int t = s; t > 1; t >>= 1) ++lg;
    return ((nout * s + 31) / 32) * (((n1 + s - 1) / s) * n2 + 4 * lg + 8);   // + 8: a round's own work
}
__host__ __device__ constexpr int digest_split(int nout, int n1, int n2) {
    int best = 1;
    for (int s = 2; s <= 32; s *= 2)
        if (s <= n1 && digest_cost(nout, n1, n2, s) < digest_cost(nout, n1, n2, best)) best = s;
    return best;
}
template <int NOUT, int N1, int N2, int ST1, int ST2, typename Base, typename Addr>
__device__ __forceinline__ void digest_group(int lane, double w, unsigned long long* A, const double* I,
                                             const double* Dv, Base base, Addr addr) {
    constexpr int S = digest_split(NOUT, N1, N2);
    constexpr int PER = 32 / S;   // outputs per round
    for (int o0 = 0; o0 < NOUT; o0 += PER) {
        const int o = o0 + lane / S, p = lane % S;
        double sum = 0.0;
        if (o < NOUT) {
            const double* row = I + base(o);
            for (int k1 = p; k1 < N1; k1 += S) {
#pragma unroll
                for (int k2 = 0; k2 < N2; ++k2) sum = fma(row[k1 * ST1 + k2 * ST2], Dv[k1 * N2 + k2], sum);
            }
        }
#pragma unroll
        for (int off = S / 2; off > 0; off >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, off, S);
        if (o < NOUT && p == 0) atomic_fixed(A + addr(o), w * sum);
    }
}

template <int La, int Lb, int Lc, int Ld>
__device__ __forceinline__ void coop_quartet(const DevData& d, int P, int Q, double* acc, double* V, double* Db,
                                             int lane, int* nq_done, int* np_done) {
    using Cls = EriClass<La, Lb, Lc, Ld>;
    using Lay = CoopLayout<La, Lb, Lc, Ld>;
    constexpr int NA = Cls::NA, NB = Cls::NB, NC = Cls::NC, ND = Cls::ND, NE = Cls::NE, NF = Cls::NF;
    constexpr int NAB = Lay::NAB, NCD = Lay::NCD, M = Cls::M;
    const int n = d.nbasis, ns = d.nshell;
    const int qa = d.pr_qa[P], qb = d.pr_qb[P], qc = d.pr_qa[Q], qd = d.pr_qb[Q];
    const int sa = d.q_parent[qa], sb = d.q_parent[qb], sc = d.q_parent[qc], sd = d.q_parent[qd];
    const double* cm = d.cutmat;
    double dnmax = fmax(4.0 * cm[sa * ns + sb], 4.0 * cm[sc * ns + sd]);
    dnmax = fmax(dnmax, fmax(cm[sa * ns + sd], cm[sa * ns + sc]));
    dnmax = fmax(dnmax, fmax(cm[sb * ns + sc], cm[sb * ns + sd]));
    const double ct = d.pr_Y[P] * d.pr_Y[Q];
    if (!(ct > d.cut) || !(ct * dnmax > d.cut)) return;   // warp-uniform
    if (lane == 0) ++*nq_done;
    const int ia = d.q_atom[qa], ib = d.q_atom[qb], ic = d.q_atom[qc], id = d.q_atom[qd];
    const double ABx = d.xyz[3 * ia] - d.xyz[3 * ib], ABy = d.xyz[3 * ia + 1] - d.xyz[3 * ib + 1],
                 ABz = d.xyz[3 * ia + 2] - d.xyz[3 * ib + 2];
    const double Cx = d.xyz[3 * ic], Cy = d.xyz[3 * ic + 1], Cz = d.xyz[3 * ic + 2];
    const double CDx = Cx - d.xyz[3 * id], CDy = Cy - d.xyz[3 * id + 1], CDz = Cz - d.xyz[3 * id + 2];

    // the six density blocks, copied into shared memory while the VRR runs
    const int fa = d.q_f0[qa], fb = d.q_f0[qb], fc = d.q_f0[qc], fd = d.q_f0[qd];
    double* Dab = Db;
    double* Dcd = Dab + NAB;
    double* Dbd = Dcd + NCD;
    double* Dad = Dbd + NB * ND;
    double* Dbc = Dad + NA * ND;
    double* Dac = Dbc + NB * NC;
    for (int t = lane; t < NAB; t += 32) cp_async8(Dab + t, d.D + (size_t)(fa + t / NB) * n + fb + t % NB);
    for (int t = lane; t < NCD; t += 32) cp_async8(Dcd + t, d.D + (size_t)(fc + t / ND) * n + fd + t % ND);
    for (int t = lane; t < NB * ND; t += 32) cp_async8(Dbd + t, d.D + (size_t)(fb + t / ND) * n + fd + t % ND);
    for (int t = lane; t < NA * ND; t += 32) cp_async8(Dad + t, d.D + (size_t)(fa + t / ND) * n + fd + t % ND);
    for (int t = lane; t < NB * NC; t += 32) cp_async8(Dbc + t, d.D + (size_t)(fb + t / NC) * n + fc + t % NC);
    for (int t = lane; t < NA * NC; t += 32) cp_async8(Dac + t, d.D + (size_t)(fa + t / NC) * n + fc + t % NC);
    cp_async_commit();

    const int mq = d.q_ltop[qa] + d.q_ltop[qb] + d.q_ltop[qc] + d.q_ltop[qd];
    coop_contract<La, Lb, Lc, Ld>(d, d.pr_pp0[P], d.pr_npp[P], d.pr_pps[P], d.pr_pp0[Q], d.pr_npp[Q], d.pr_pps[Q],
                                  Cx, Cy, Cz, dnmax, true, mq, acc, V, lane, np_done);
    __syncwarp();   // acc complete (also when every primitive quartet was screened out)
    // bra HRR (one ket column per lane), then ket HRR (one bra row per lane)
    double* t1 = V;
    double* I = V + NF * NAB;
    for (int f = lane; f < NF; f += 32) Cls::hrr_bra(acc + f * NE, t1 + f * NAB, ABx, ABy, ABz);
    __syncwarp();
    // ket HRR one bra row per lane, the row scaled by QUICK's cons factors as it is written
    for (int ab = lane; ab < NAB; ab += 32) {
        double* row = I + ab * NCD;
        Cls::hrr_ket(t1 + ab, NAB, row, CDx, CDy, CDz);
        const double cab = Cls::cons_a(ab / NB) * Cls::cons_b(ab % NB);
        for (int cd = 0; cd < NCD; ++cd) row[cd] *= cab * Cls::cons_c(cd / ND) * Cls::cons_d(cd % ND);
    }
    cp_async_wait_all();
    __syncwarp();
    const double deg = (qa != qb ? 2.0 : 1.0) * (qc != qd ? 2.0 : 1.0) * (P != Q ? 2.0 : 1.0);
    const double wJ = 0.25 * deg, wK = -0.0625 * deg;
    unsigned long long* A = d.A;
    // J over the bra: (ab) row . Dcd;  J over the ket: (cd) column . Dab
    if (!d.exchange_only) {   // warp-uniform
        digest_group<NAB, NC, ND, ND, 1>(
            lane, wJ, A, I, Dcd, [&](int ab) { return ab * NCD; },
            [&](int ab) { return (size_t)(fa + ab / NB) * n + fb + ab % NB; });
        digest_group<NCD, NA, NB, NB * NCD, NCD>(
            lane, wJ, A, I, Dab, [&](int cd) { return cd; },
            [&](int cd) { return (size_t)(fc + cd / ND) * n + fd + cd % ND; });
    }
    // K_ac = sum_bd I D_bd,  K_bc = sum_ad I D_ad,  K_ad = sum_bc I D_bc,  K_bd = sum_ac I D_ac
    digest_group<NA * NC, NB, ND, NCD, 1>(
        lane, wK, A, I, Dbd, [&](int ac) { return (ac / NC) * NB * NCD + (ac % NC) * ND; },
        [&](int ac) { return (size_t)(fa + ac / NC) * n + fc + ac % NC; });
    digest_group<NB * NC, NA, ND, NB * NCD, 1>(
        lane, wK, A, I, Dad, [&](int bc) { return (bc / NC) * NCD + (bc % NC) * ND; },
        [&](int bc) { return (size_t)(fb + bc / NC) * n + fc + bc % NC; });
    digest_group<NA * ND, NB, NC, NCD, ND>(
        lane, wK, A, I, Dbc, [&](int ad) { return (ad / ND) * NB * NCD + ad % ND; },
        [&](int ad) { return (size_t)(fa + ad / ND) * n + fd + ad % ND; });
    digest_group<NB * ND, NA, NC, NB * NCD, ND>(
        lane, wK, A, I, Dac, [&](int bd) { return (bd / ND) * NCD + bd % ND; },
        [&](int bd) { return (size_t)(fb + bd / ND) * n + fd + bd % ND; });
    __syncwarp();
}

constexpr int kCoopWarps = 4;   // largest warps-per-block of a cooperative class

template <int La, int Lb, int Lc, int Ld>
__global__ void __launch_bounds__(32 * kCoopWarps)
fock_coop_kernel(DevData d, const int4* __restrict__ items, int n_items, int* __restrict__ counter) {
    using Lay = CoopLayout<La, Lb, Lc, Ld>;
    extern __shared__ double smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double* acc = smem + (size_t)warp * Lay::PER_WARP;
    double* V = acc + Lay::ACC;
    double* Db = V + Lay::WORK;
    for (;;) {
        int it = 0;
        if (lane == 0) it = atomicAdd(counter, 1);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= n_items) break;
        const int4 w = items[it];
        int nq = 0, np = 0;
        for (int k = 0; k < w.z; ++k) coop_quartet<La, Lb, Lc, Ld>(d, w.x, w.y + k, acc, V, Db, lane, &nq, &np);
        if (d.stats && lane == 0) {
            atomicAdd(d.stats, (unsigned long long)nq);
            atomicAdd(d.stats + 1, (unsigned long long)np);
        }
    }
}

// The class's Boys row table (kBoysNT rows of 64 bytes): an evaluation reads one
// row with four 16-byte loads, served from L1 for the hot part of the T range.
// (Staging the 46 KB table in shared memory costs more in occupancy than it
// saves in load latency: measured 1.8x slower on the ssss class.)
template <int M>
__device__ __forceinline__ const double2* class_boys_rows(const double2* __restrict__ src) {
    return src + (size_t)M * kBoysNT * (kBoysRow / 2);
}

// Per-lane class kernels launch with 1..kMaxLaneWarps warps per block (default
// kWarpsPerBlock; the autotuner picks per class).  Their register ceiling is the
// class's LANE_REGS (gen_eri.py: measured per class; 255 = ptxas's own choice, which
// 256-thread blocks can always launch).
constexpr int kMaxLaneWarps = 8;

// Work item: x = bra pair, y = first ket pair, z = number of kets (<= 32),
// w = 1 for the mixed form's FP32 quartets.
// FP32 = true: the mixed form's small-bound items (VRR and contraction in FP32),
// compiled apart so that the FP64 items keep their register budget and vice versa.
// One work item of a per-lane class (the warp's bra pair against up to 32 kets,
// one quartet per lane), J of the bra pair summed over the warp.
template <int La, int Lb, int Lc, int Ld, bool FP32>
__device__ __forceinline__ void lane_item(const DevData& d, const double2* __restrict__ bt, const int4 w,
                                          int lane) {
    using Cls = EriClass<La, Lb, Lc, Ld>;
    constexpr int NAB = Cls::NA * Cls::NB;
    double jab[NAB];
#pragma unroll
    for (int i = 0; i < NAB; ++i) jab[i] = 0.0;
    int nq = 0, np = 0;
    if (lane < w.z) fock_quartet<La, Lb, Lc, Ld, FP32>(d, bt, w.x, w.y + lane, jab, &nq, &np);
    if (d.stats) {
        const unsigned sq = __reduce_add_sync(0xffffffffu, (unsigned)nq);
        const unsigned sp = __reduce_add_sync(0xffffffffu, (unsigned)np);
        if (lane == 0) {
            atomicAdd(d.stats, (unsigned long long)sq);
            atomicAdd(d.stats + 1, (unsigned long long)sp);
        }
    }
    if (d.exchange_only) return;   // no J part
    const int P = w.x;
    const int qa = d.pr_qa[P], qb = d.pr_qb[P];
    const int fa = d.q_f0[qa], fb = d.q_f0[qb];
#pragma unroll
    for (int i = 0; i < NAB; ++i) {
        const double s = warp_sum(jab[i]);
        if (lane == 0 && s != 0.0)
            atomic_fixed(d.A + (size_t)(fa + i / Cls::NB) * d.nbasis + fb + i % Cls::NB, s);
    }
}

template <int La, int Lb, int Lc, int Ld, bool FP32>
__global__ void __maxnreg__((EriClass<La, Lb, Lc, Ld>::LANE_REGS))
fock_class_kernel(DevData d, const int4* __restrict__ items, int n_items, int* __restrict__ counter) {
    using Cls = EriClass<La, Lb, Lc, Ld>;
    const int lane = threadIdx.x & 31;
    const double2* bt = class_boys_rows<Cls::M>(d.boys8);
    for (;;) {
        int it = 0;
        if (lane == 0) it = atomicAdd(counter, 1);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= n_items) break;
        lane_item<La, Lb, Lc, Ld, FP32>(d, bt, items[it], lane);
    }
}

// The s/p classes in one persistent kernel (qk_set_merge_sp): the six per-lane s/p
// classes' item lists joined into one virtual list, heaviest class first, walked
// with one atomic counter; a warp finds its item's class by binary search over the
// segments' prefix counts and runs that class's straight-line code.  One launch
// instead of six, at the register allocation of the largest of the six.
struct MergedSeg {
    const int4* items;
    int begin;   // items of the joined list before this segment
    int cls;     // position in kSpMerged
};
constexpr int kSpMergedN = 6;
constexpr int kSpMerged[kSpMergedN][4] = {{1, 1, 1, 1}, {1, 1, 1, 0}, {1, 1, 0, 0}, {1, 0, 1, 0}, {1, 0, 0, 0},
                                          {0, 0, 0, 0}};

#if QK_MAX_L >= 1
template <bool FP32>
__global__ void __launch_bounds__(32 * kMaxLaneWarps)
fock_merged_sp_kernel(DevData d, const MergedSeg* __restrict__ segs, int nseg, int n_items,
                      int* __restrict__ counter) {
    const int lane = threadIdx.x & 31;
    for (;;) {
        int it = 0;
        if (lane == 0) it = atomicAdd(counter, 1);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= n_items) break;
        int lo = 0, hi = nseg - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (segs[mid].begin <= it) lo = mid; else hi = mid - 1;
        }
        const MergedSeg sg = segs[lo];
        const int4 w = sg.items[it - sg.begin];
        switch (sg.cls) {
            case 0: lane_item<1, 1, 1, 1, FP32>(d, class_boys_rows<EriClass<1, 1, 1, 1>::M>(d.boys8), w, lane); break;
            case 1: lane_item<1, 1, 1, 0, FP32>(d, class_boys_rows<EriClass<1, 1, 1, 0>::M>(d.boys8), w, lane); break;
            case 2: lane_item<1, 1, 0, 0, FP32>(d, class_boys_rows<EriClass<1, 1, 0, 0>::M>(d.boys8), w, lane); break;
            case 3: lane_item<1, 0, 1, 0, FP32>(d, class_boys_rows<EriClass<1, 0, 1, 0>::M>(d.boys8), w, lane); break;
            case 4: lane_item<1, 0, 0, 0, FP32>(d, class_boys_rows<EriClass<1, 0, 0, 0>::M>(d.boys8), w, lane); break;
            default: lane_item<0, 0, 0, 0, FP32>(d, class_boys_rows<EriClass<0, 0, 0, 0>::M>(d.boys8), w, lane); break;
        }
    }
}
#endif


// Batched (many-molecule) variants.  Per class, the work of every molecule stays
// in that molecule's own item list; a segment table (one entry per molecule with
// work in the class: its list, the prefix count of items before it, its index)
// joins them into one virtual list that the warps walk with one atomic counter.
// A warp finds the segment of its item by binary search over the prefix counts
// (a few cached loads, shared by the warp) -- nothing is copied or re-sorted
// when molecules join or leave the batch.
struct BatchSeg {
    const int4* items;
    int begin;   // items of the class before this segment
    int mol;     // index into the batch's DevData array
};

__device__ __forceinline__ int batch_find_seg(const BatchSeg* __restrict__ segs, int nseg, int it) {
    int lo = 0, hi = nseg - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (segs[mid].begin <= it) lo = mid; else hi = mid - 1;
    }
    return lo;
}

template <int La, int Lb, int Lc, int Ld, bool FP32>
__global__ void __maxnreg__((EriClass<La, Lb, Lc, Ld>::LANE_REGS))
fock_class_kernel_batch(const DevData* __restrict__ dl, const BatchSeg* __restrict__ segs, int nseg, int n_items,
                        int* __restrict__ counter) {
    using Cls = EriClass<La, Lb, Lc, Ld>;
    constexpr int NAB = Cls::NA * Cls::NB;
    const int lane = threadIdx.x & 31;
    const double2* bt = class_boys_rows<Cls::M>(dl[0].boys8);
    for (;;) {
        int it = 0;
        if (lane == 0) it = atomicAdd(counter, 1);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= n_items) break;
        const BatchSeg sg = segs[batch_find_seg(segs, nseg, it)];
        const int4 w = sg.items[it - sg.begin];
        const DevData& d = dl[sg.mol];
        double jab[NAB];
#pragma unroll
        for (int i = 0; i < NAB; ++i) jab[i] = 0.0;
        int nq = 0, np = 0;
        if (lane < w.z) fock_quartet<La, Lb, Lc, Ld, FP32>(d, bt, w.x, w.y + lane, jab, &nq, &np);
        if (d.exchange_only) continue;
        const int P = w.x;
        const int fa = d.q_f0[d.pr_qa[P]], fb = d.q_f0[d.pr_qb[P]];
#pragma unroll
        for (int i = 0; i < NAB; ++i) {
            const double s = warp_sum(jab[i]);
            if (lane == 0 && s != 0.0)
                atomic_fixed(d.A + (size_t)(fa + i / Cls::NB) * d.nbasis + fb + i % Cls::NB, s);
        }
    }
}

template <int La, int Lb, int Lc, int Ld>
__global__ void __launch_bounds__(32 * kCoopWarps)
fock_coop_kernel_batch(const DevData* __restrict__ dl, const BatchSeg* __restrict__ segs, int nseg, int n_items,
                       int* __restrict__ counter) {
    using Lay = CoopLayout<La, Lb, Lc, Ld>;
    extern __shared__ double smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double* acc = smem + (size_t)warp * Lay::PER_WARP;
    double* V = acc + Lay::ACC;
    double* Db = V + Lay::WORK;
    for (;;) {
        int it = 0;
        if (lane == 0) it = atomicAdd(counter, 1);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= n_items) break;
        const BatchSeg sg = segs[batch_find_seg(segs, nseg, it)];
        const int4 w = sg.items[it - sg.begin];
        const DevData& d = dl[sg.mol];
        int nq = 0, np = 0;
        for (int k = 0; k < w.z; ++k) coop_quartet<La, Lb, Lc, Ld>(d, w.x, w.y + k, acc, V, Db, lane, &nq, &np);
    }
}

// The per-lane kernels of the s/p classes, single-molecule and batched, FP64 and FP32.
// When the build compiles them in their own translation unit (fock_lane_sp.cu,
// QK_LANE_SP_TU_SEPARATE), this unit only declares them.
#define QK_LANE_SP_CLASSES(X) X(0, 0, 0, 0) X(1, 0, 0, 0) X(1, 0, 1, 0) X(1, 1, 0, 0) X(1, 1, 1, 0) X(1, 1, 1, 1)
#if defined(QK_LANE_SP_TU_SEPARATE) && !defined(QK_LANE_SP_TU) && QK_MAX_L >= 1
#define QK_LANE_SP_EXTERN(a, b, c, e)                                                                     \
    extern template __global__ void fock_class_kernel<a, b, c, e, false>(DevData, const int4*, int, int*); \
    extern template __global__ void fock_class_kernel<a, b, c, e, true>(DevData, const int4*, int, int*);  \
    extern template __global__ void fock_class_kernel_batch<a, b, c, e, false>(const DevData*, const BatchSeg*, \
                                                                               int, int, int*);             \
    extern template __global__ void fock_class_kernel_batch<a, b, c, e, true>(const DevData*, const BatchSeg*,  \
                                                                              int, int, int*);
QK_LANE_SP_CLASSES(QK_LANE_SP_EXTERN)
#undef QK_LANE_SP_EXTERN
#endif

#ifdef QK_LANE_SP_TU
}  // namespace qk
#else

// Per-molecule set-up and finish of a batched build, one launch each for all
// molecules: grid (chunks, molecules), grid-stride inside a molecule.
struct BatchMol {
    const double* D;
    double* cut;                  // density screen to compute here, or null (caller's)
    unsigned long long* A;
    double* o;
    const int* s_f0;
    const int* s_f1;
    int n, ns;
};

__global__ void batch_prep_kernel(const BatchMol* __restrict__ ml) {
    const BatchMol m = ml[blockIdx.y];
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long t0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nn = (long long)m.n * m.n;
    for (long long t = t0; t < nn; t += stride) m.A[t] = 0ull;
    if (m.cut) {
        const long long ns2 = (long long)m.ns * m.ns;
        for (long long t = t0; t < ns2; t += stride) {
            const int a = (int)(t / m.ns), b = (int)(t % m.ns);
            double v = 0.0;
            for (int i = m.s_f0[a]; i < m.s_f1[a]; ++i)
                for (int j = m.s_f0[b]; j < m.s_f1[b]; ++j) v = fmax(v, fabs(m.D[(size_t)j * m.n + i]));
            m.cut[t] = v;
        }
    }
}

__global__ void batch_finalize_kernel(const BatchMol* __restrict__ ml) {
    const BatchMol m = ml[blockIdx.y];
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long nn = (long long)m.n * m.n;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nn; t += stride) {
        const int i = (int)(t / m.n), j = (int)(t % m.n);
        const long long v = (long long)(m.A[(size_t)i * m.n + j] + m.A[(size_t)j * m.n + i]);
        m.o[t] += (double)v * kFixedInv;
    }
}

// Schwarz bounds: one thread per (pair, mode); mode < 0 = contracted (ab|ab),
// mode = k = primitive-pair diagonal quartet of primitive pair k.  Writes
// max |(ab|ab)| (with QUICK's cons factors) through an unsigned atomicMax on the
// bit pattern (valid for non-negative doubles).
template <int La, int Lb>
__global__ void __launch_bounds__(128)
schwarz_kernel(DevData d, const int2* __restrict__ work, int n_work, const int* __restrict__ q_prim0,
               const int* __restrict__ q_nprim,
               int nshell, int jbasis, unsigned long long* __restrict__ Ysq,
               unsigned long long* __restrict__ cpsq) {
    using Cls = EriClass<La, Lb, La, Lb>;
    constexpr int NA = Cls::NA, NB = Cls::NB, NE = Cls::NE, NF = Cls::NF, NAB = NA * NB;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_work) return;
    const int P = work[t].x, mode = work[t].y;
    const int qa = d.pr_qa[P], qb = d.pr_qb[P];
    const int ia = d.q_atom[qa], ib = d.q_atom[qb];
    const double AB[3] = {d.xyz[3 * ia] - d.xyz[3 * ib], d.xyz[3 * ia + 1] - d.xyz[3 * ib + 1],
                          d.xyz[3 * ia + 2] - d.xyz[3 * ib + 2]};
    const double Cc[3] = {d.xyz[3 * ia], d.xyz[3 * ia + 1], d.xyz[3 * ia + 2]};
    int p0 = d.pr_pp0[P], np = d.pr_npp[P];
    const int ps = d.pr_pps[P];
    if (mode >= 0) { p0 += mode * ps; np = 1; }
    double acc[NE * NF];
    int ndone = 0;
    contract_quartet<La, Lb, La, Lb>(d, d.boys8 + (size_t)Cls::M * kBoysNT * (kBoysRow / 2), p0, np, ps, p0, np, ps,
                                     Cc, 0.0, false, 2 * (d.q_ltop[qa] + d.q_ltop[qb]), acc, &ndone);
    double t1[NF * NAB];
#pragma unroll
    for (int f = 0; f < NF; ++f) Cls::hrr_bra(acc + f * NE, t1 + f * NAB, AB[0], AB[1], AB[2]);
    double ymax = 0.0;
#pragma unroll
    for (int a = 0; a < NA; ++a)
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const int ab = a * NB + b;
            double I[NAB];
            Cls::hrr_ket(t1 + ab, NAB, I, AB[0], AB[1], AB[2]);
            const double c = Cls::cons_a(a) * Cls::cons_b(b);
            ymax = fmax(ymax, fabs(I[ab] * c * c));
        }
    const unsigned long long bits = (unsigned long long)__double_as_longlong(ymax);
    if (mode < 0) {
        const int sa = d.q_parent[qa], sb = d.q_parent[qb];
        atomicMax(Ysq + (size_t)sa * nshell + sb, bits);
        atomicMax(Ysq + (size_t)sb * nshell + sa, bits);
    } else {
        // QUICK's cutprim squares X0*Xcoeff (classprim, src/modules/quick_cutoff_module.f90:448-457),
        // so cutprim^2 = X0 * (ij|ij)_prim; reproduce that definition.
        const unsigned long long pbits = (unsigned long long)__double_as_longlong(ymax * kX0);
        // primitive pair k of a pair is (i, j) with k = i * nprim(qb) + j
        const int nbp = q_nprim[qb];
        const int gi = q_prim0[qa] + mode / nbp, gj = q_prim0[qb] + mode % nbp;
        atomicMax(cpsq + (size_t)gi * jbasis + gj, pbits);
        atomicMax(cpsq + (size_t)gj * jbasis + gi, pbits);
    }
}

// Schwarz bounds for the cooperative classes: one warp per (pair, mode), the
// contraction of coop_contract without screening, HRR as in coop_quartet, and
// the largest diagonal integral |(ab|ab)| of the pair block.
template <int La, int Lb>
__global__ void __launch_bounds__(32 * kCoopWarps)
schwarz_coop_kernel(DevData d, const int2* __restrict__ work, int n_work, const int* __restrict__ q_prim0,
                    const int* __restrict__ q_nprim, int nshell, int jbasis, unsigned long long* __restrict__ Ysq,
                    unsigned long long* __restrict__ cpsq) {
    using Cls = EriClass<La, Lb, La, Lb>;
    using Lay = CoopLayout<La, Lb, La, Lb>;
    constexpr int NB = Cls::NB, NE = Cls::NE, NF = Cls::NF, NAB = Lay::NAB, NCD = Lay::NCD;
    extern __shared__ double smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    double* acc = smem + (size_t)warp * Lay::PER_WARP;
    double* V = acc + Lay::ACC;
    for (int t = blockIdx.x * wpb + warp; t < n_work; t += gridDim.x * wpb) {
        const int P = work[t].x, mode = work[t].y;
        const int qa = d.pr_qa[P], qb = d.pr_qb[P];
        const int ia = d.q_atom[qa], ib = d.q_atom[qb];
        const double ABx = d.xyz[3 * ia] - d.xyz[3 * ib], ABy = d.xyz[3 * ia + 1] - d.xyz[3 * ib + 1],
                     ABz = d.xyz[3 * ia + 2] - d.xyz[3 * ib + 2];
        int p0 = d.pr_pp0[P], np = d.pr_npp[P];
        const int ps = d.pr_pps[P];
        if (mode >= 0) { p0 += mode * ps; np = 1; }
        int ndone = 0;
        coop_contract<La, Lb, La, Lb>(d, p0, np, ps, p0, np, ps, d.xyz[3 * ia], d.xyz[3 * ia + 1],
                                      d.xyz[3 * ia + 2], 0.0, false, 2 * (d.q_ltop[qa] + d.q_ltop[qb]), acc, V, lane,
                                      &ndone);
        __syncwarp();
        double* t1 = V;
        double* I = V + NF * NAB;
        for (int f = lane; f < NF; f += 32) Cls::hrr_bra(acc + f * NE, t1 + f * NAB, ABx, ABy, ABz);
        __syncwarp();
        double ymax = 0.0;
        for (int ab = lane; ab < NAB; ab += 32) {
            Cls::hrr_ket(t1 + ab, NAB, I + ab * NCD, ABx, ABy, ABz);
            const double c = Cls::cons_a(ab / NB) * Cls::cons_b(ab % NB);
            ymax = fmax(ymax, fabs(I[ab * NCD + ab] * c * c));
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) ymax = fmax(ymax, __shfl_xor_sync(0xffffffffu, ymax, o));
        if (lane == 0) {
            if (mode < 0) {
                const unsigned long long bits = (unsigned long long)__double_as_longlong(ymax);
                const int sa = d.q_parent[qa], sb = d.q_parent[qb];
                atomicMax(Ysq + (size_t)sa * nshell + sb, bits);
                atomicMax(Ysq + (size_t)sb * nshell + sa, bits);
            } else {
                // QUICK's cutprim: cutprim^2 = X0 * (ij|ij)_prim (see schwarz_kernel)
                const unsigned long long pbits = (unsigned long long)__double_as_longlong(ymax * kX0);
                const int nbp = q_nprim[qb];
                const int gi = q_prim0[qa] + mode / nbp, gj = q_prim0[qb] + mode % nbp;
                atomicMax(cpsq + (size_t)gi * jbasis + gj, pbits);
                atomicMax(cpsq + (size_t)gj * jbasis + gi, pbits);
            }
        }
        __syncwarp();
    }
}

// Launch the Schwarz kernel of pair class (a, b): per-thread for the small
// classes, warp-cooperative for the large ones.
template <int a, int b>
static cudaError_t launch_schwarz(const DevData& d, const int2* wl, int n, const int* q_prim0, const int* q_nprim,
                                  int ns, int jb, unsigned long long* Ysq, unsigned long long* cpsq, int num_sms,
                                  cudaStream_t s) {
    if constexpr (EriClass<a, b, a, b>::COOP) {
        using Lay = CoopLayout<a, b, a, b>;
        const size_t smem = sizeof(double) * Lay::WARPS * Lay::PER_WARP;
        if (smem > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute((const void*)&schwarz_coop_kernel<a, b>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
        }
        const int grid = std::min((n + Lay::WARPS - 1) / Lay::WARPS, num_sms * 8);
        schwarz_coop_kernel<a, b><<<grid, 32 * Lay::WARPS, smem, s>>>(d, wl, n, q_prim0, q_nprim, ns, jb, Ysq, cpsq);
    } else {
        schwarz_kernel<a, b><<<(n + 127) / 128, 128, 0, s>>>(d, wl, n, q_prim0, q_nprim, ns, jb, Ysq, cpsq);
    }
    return cudaGetLastError();
}

__global__ void density_cutoff_kernel(const double* __restrict__ D, int n, int nshell,
                                      const int* __restrict__ s_f0, const int* __restrict__ s_f1,
                                      double* __restrict__ cutmat) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nshell * nshell) return;
    const int a = t / nshell, b = t % nshell;
    double m = 0.0;
    for (int i = s_f0[a]; i < s_f1[a]; ++i)
        for (int j = s_f0[b]; j < s_f1[b]; ++j) m = fmax(m, fabs(D[(size_t)j * n + i]));
    cutmat[t] = m;
}

// FP64 FMA throughput probe: independent dependent-chains per thread.
__global__ void fp64_probe_kernel(double* out, int iters, double a, double b) {
    double x0 = threadIdx.x * 1e-3, x1 = x0 + 1.0, x2 = x0 + 2.0, x3 = x0 + 3.0;
    double x4 = x0 + 4.0, x5 = x0 + 5.0, x6 = x0 + 6.0, x7 = x0 + 7.0;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
            x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
        }
    }
    const double r = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (r == 12345.678) out[0] = r;   // keeps the chains live
}

// Boys function probe: F_0..F_M at each T by the two device forms the Fock
// kernels use -- the per-lane row-table evaluation (boys_scaled_rows<M>, scale 1)
// and the cooperative kernels' one-m evaluation (boys_one) -- for testing them
// directly against high-precision values.
template <int M>
__global__ void boys_probe_kernel(const double* __restrict__ T, int n, const double2* __restrict__ rows8,
                                  const double* __restrict__ tab, int mode, double* __restrict__ f_rows,
                                  double* __restrict__ f_one) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double F[M + 1];
    if (mode)
        boys_quick_scaled<M>(T[i], 1.0, F, M);
    else
        boys_scaled_rows<M>(T[i], 1.0, rows8 + (size_t)M * kBoysNT * (kBoysRow / 2), F);
#pragma unroll
    for (int m = 0; m <= M; ++m) {
        f_rows[(size_t)i * (M + 1) + m] = F[m];
        f_one[(size_t)i * (M + 1) + m] = mode ? boys_quick_one(m, M, T[i]) : boys_one(m, T[i], tab);
    }
}

template <int M>
static cudaError_t launch_boys_probe(const double* T, int n, const double2* rows8, const double* tab, int mode,
                                     double* fr, double* fo, cudaStream_t s) {
    boys_probe_kernel<M><<<(n + 127) / 128, 128, 0, s>>>(T, n, rows8, tab, mode, fr, fo);
    return cudaGetLastError();
}

// Open shell (UHF): total and spin densities Dt = Da + Db, Ds = Da - Db.
__global__ void uhf_densities_kernel(const double* __restrict__ Da, const double* __restrict__ Db, long long nn,
                                     double* __restrict__ Dt, double* __restrict__ Ds) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nn; t += (long long)gridDim.x * blockDim.x) {
        const double a = Da[t], b = Db[t];
        Dt[t] = a + b;
        Ds[t] = a - b;
    }
}

// QUICK's open-shell density screen (oshell_density_cutoff, src/modules/include/cutoff.fh:15-92):
// per shell pair the largest of |Da + Db|, |Da|, |Db| over its block.
__global__ void density_cutoff_uhf_kernel(const double* __restrict__ Da, const double* __restrict__ Db, int n,
                                          int nshell, const int* __restrict__ s_f0, const int* __restrict__ s_f1,
                                          double* __restrict__ cutmat) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nshell * nshell) return;
    const int a = t / nshell, b = t % nshell;
    double m = 0.0;
    for (int i = s_f0[a]; i < s_f1[a]; ++i)
        for (int j = s_f0[b]; j < s_f1[b]; ++j) {
            const double x = Da[(size_t)j * n + i], y = Db[(size_t)j * n + i];
            m = fmax(m, fmax(fabs(x + y), fmax(fabs(x), fabs(y))));
        }
    cutmat[t] = m;
}

// oa += G_cs(Dt) + K(Ds), ob += G_cs(Dt) - K(Ds): A1 the closed-shell build of Dt,
// A2 the exchange-only build of Ds (both int64 fixed point; sums taken exactly).
__global__ void finalize_uhf_kernel(const unsigned long long* __restrict__ A1, const unsigned long long* __restrict__ A2,
                                    int n, double* __restrict__ oa, double* __restrict__ ob) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * n) return;
    const int i = t / n, j = t % n;
    const size_t ij = (size_t)i * n + j, ji = (size_t)j * n + i;
    const unsigned long long j1 = A1[ij] + A1[ji], k2 = A2[ij] + A2[ji];
    oa[t] += (double)(long long)(j1 + k2) * kFixedInv;
    ob[t] += (double)(long long)(j1 - k2) * kFixedInv;
}

__global__ void finalize_kernel(const unsigned long long* __restrict__ A, int n, double* __restrict__ o) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * n) return;
    const int i = t / n, j = t % n;
    const long long s = (long long)(A[(size_t)i * n + j] + A[(size_t)j * n + i]);
    o[t] += (double)s * kFixedInv;
}

}  // namespace qk

// =========================================================================== host
namespace qk {


template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0, cap = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { if (p) cudaFree(p); }
    // Grows by at least a quarter when it grows: a context reused for a slightly
    // larger molecule then keeps its buffers (cudaFree synchronises the whole GPU).
    cudaError_t reserve(size_t count) {
        n = count;
        if (count <= cap && p) return cudaSuccess;
        const size_t want = cap > 0 ? std::max(count, cap + cap / 4) : count;
        if (p) { cudaFree(p); p = nullptr; cap = 0; }
        if (count == 0) return cudaSuccess;
        cudaError_t e = cudaMalloc(&p, want * sizeof(T));
        if (e == cudaSuccess) cap = want;
        return e;
    }
    size_t bytes() const { return cap * sizeof(T); }
    cudaError_t upload(const std::vector<T>& v, cudaStream_t s) {
        cudaError_t e = reserve(v.size());
        if (e != cudaSuccess || v.empty()) return e;
        return cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s);
    }
};

constexpr int kMaxPrimShell = 32;

struct Qsh {
    int L, parent, atom, nprim, prim0, f0;
    double coef[kMaxPrimShell], expo[kMaxPrimShell];
};

struct Bucket {
    int La, Lb, npa, npb, begin, end;
};

// Primitive-pair data is stored bucket-interleaved: primitive pair k of pair P sits
// at pp0[P] + k * pps[P] with pps = bucket size, so the 32 consecutive ket pairs of
// a warp item read consecutive addresses (coalesced).
struct PairTable {
    std::vector<int> qa, qb, pp0, npp, pps;
    std::vector<double> Y;
    std::vector<double2> zo, kc, pxy, pzax, payz;   // the five 16-byte fields of DevData
    std::vector<Bucket> buckets;
    DevBuf<int> d_qa, d_qb, d_pp0, d_npp, d_pps, d_lt;
    DevBuf<double> d_Y;
    DevBuf<double2> d_zo, d_kc, d_pxy, d_pzax, d_payz, d_geo;
    DevBuf<int4> d_sh;
    void clear() {
        qa.clear(); qb.clear(); pp0.clear(); npp.clear(); pps.clear(); Y.clear();
        zo.clear(); kc.clear(); pxy.clear(); pzax.clear(); payz.clear(); buckets.clear();
    }
};

using FockFn = void (*)(bool, dim3, dim3, size_t, cudaStream_t, const DevData&, const int4*, int, int*);
template <int a, int b, int c, int e>
void launch_fock(bool fp32, dim3 g, dim3 bl, size_t smem, cudaStream_t s, const DevData& dd, const int4* it, int n,
                 int* cnt) {
    if constexpr (EriClass<a, b, c, e>::COOP)
        fock_coop_kernel<a, b, c, e><<<g, bl, smem, s>>>(dd, it, n, cnt);
    else if (fp32)
        fock_class_kernel<a, b, c, e, true><<<g, bl, smem, s>>>(dd, it, n, cnt);
    else
        fock_class_kernel<a, b, c, e, false><<<g, bl, smem, s>>>(dd, it, n, cnt);
}
template <int a, int b, int c, int e>
const void* fock_fn_ptr(bool fp32) {
    if constexpr (EriClass<a, b, c, e>::COOP)
        return (const void*)&fock_coop_kernel<a, b, c, e>;
    else if (fp32)
        return (const void*)&fock_class_kernel<a, b, c, e, true>;
    else
        return (const void*)&fock_class_kernel<a, b, c, e, false>;
}
using FockBatchFn = void (*)(bool, dim3, dim3, size_t, cudaStream_t, const DevData*, const BatchSeg*, int, int, int*);
template <int a, int b, int c, int e>
void launch_fock_batch(bool fp32, dim3 g, dim3 bl, size_t smem, cudaStream_t s, const DevData* dl,
                       const BatchSeg* segs, int nseg, int n, int* cnt) {
    if constexpr (EriClass<a, b, c, e>::COOP)
        fock_coop_kernel_batch<a, b, c, e><<<g, bl, smem, s>>>(dl, segs, nseg, n, cnt);
    else if (fp32)
        fock_class_kernel_batch<a, b, c, e, true><<<g, bl, smem, s>>>(dl, segs, nseg, n, cnt);
    else
        fock_class_kernel_batch<a, b, c, e, false><<<g, bl, smem, s>>>(dl, segs, nseg, n, cnt);
}
template <int a, int b, int c, int e>
const void* fock_batch_fn_ptr(bool fp32) {
    if constexpr (EriClass<a, b, c, e>::COOP)
        return (const void*)&fock_coop_kernel_batch<a, b, c, e>;
    else if (fp32)
        return (const void*)&fock_class_kernel_batch<a, b, c, e, true>;
    else
        return (const void*)&fock_class_kernel_batch<a, b, c, e, false>;
}
template <int a, int b, int c, int e>
constexpr size_t coop_smem() {
    if constexpr (EriClass<a, b, c, e>::COOP)
        return sizeof(double) * CoopLayout<a, b, c, e>::WARPS * CoopLayout<a, b, c, e>::PER_WARP;
    else
        return 0;
}

struct ClassEntry {
    int La, Lb, Lc, Ld;
    FockFn fn;
    const void* (*kernel)(bool fp32);
    double prim_flops, quartet_flops;   // algorithmic FP64 operations (gen_eri.py model)
    bool coop;                          // one quartet per warp (high angular momentum)
    size_t smem;                        // dynamic shared memory of a block (coop only)
    int coop_warps;                     // warps per block of the cooperative kernel
    FockBatchFn fn_batch;               // many-molecule variant
    const void* (*kernel_batch)(bool fp32);
};
template <int a, int b, int c, int e>
constexpr int coop_warps() {
    if constexpr (EriClass<a, b, c, e>::COOP)
        return CoopLayout<a, b, c, e>::WARPS;
    else
        return 0;
}
#define QK_X(a, b, c, e) {a, b, c, e, &launch_fock<a, b, c, e>, &fock_fn_ptr<a, b, c, e>, \
                          EriClass<a, b, c, e>::PRIM_FLOPS, EriClass<a, b, c, e>::QUARTET_FLOPS, \
                          EriClass<a, b, c, e>::COOP, coop_smem<a, b, c, e>(), coop_warps<a, b, c, e>(), \
                          &launch_fock_batch<a, b, c, e>, &fock_batch_fn_ptr<a, b, c, e>},
static const ClassEntry g_classes[] = {QK_ERI_CLASS_LIST(QK_X)};
#undef QK_X
constexpr int kNumClasses = sizeof(g_classes) / sizeof(g_classes[0]);

struct ClassWork {
    std::vector<int4> items;      // host builder only (sharded contexts)
    const int4* d_items = nullptr;   // this class's items inside the context's item buffer
    int n_items = 0;
    long long nquart = 0, nprimq = 0, nquart32 = 0;
    int block = 0;        // threads per block of the class launch
    size_t smem = 0;      // dynamic shared memory of a block
    int n64 = 0;          // items [0, n64) are FP64, [n64, size) the mixed form's FP32 ones
    int grid32 = 0;       // grid of the FP32 launch
    int grid = 0;
};

}  // namespace qk

struct qk_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::mutex mu;
    int maxprim = 20;
    int natom = 0, nbasis = 0, nshell = 0, jbasis = 0;
    std::vector<double> xyz;
    std::vector<qk::Qsh> qsh;
    std::vector<int> q_ltop_h;          // per Qshell: the top angular momentum of its shell (1 for SP)
    std::vector<int> shell_f0, shell_f1, shell_prim0;
    bool have_basis = false, have_schwarz = false;
    std::vector<double> Ycut, cutprim;   // nshell^2, jbasis^2 (symmetric)
    double integralCutoff = 1e-7, primLimit = 1e-8;
    double fp32_bound = 0.0;          // mixed form: FP32 below this Schwarz bound product
    int boys_mode = 0;                // qk_set_boys: 0 tabulated; 1 QUICK's CPU order; 2 its GPU order
    int nstreams = 4;                 // class kernels run over this many streams (0: one after another)
    int shard_rank = 0, shard_count = 1;   // this context's share of the work items (qk_set_shard)
    int cls_wpb[qk::kNumClasses] = {};    // warps per block of each class launch (0: default)
    int cls_bpsm[qk::kNumClasses] = {};   // cap on resident blocks per SM (0: as many as fit)
    double built_fp32 = -1.0;
    double built_cut = -1.0;
    bool pairs_dirty = true;
    qk::PairTable pairs;
    qk::ClassWork work[qk::kNumClasses];
    qk::DevBuf<int4> d_items;          // every class's work items, class after class
    qk::DevBuf<char> d_wl;             // scratch of the device work-list builder
    bool worklist_on_device = true;    // qk_set_worklist_builder
    int launches = 0;
    // qk_set_merge_sp: the s/p classes in one launch per precision
    bool merge_sp = false;
    bool m_ready = false;              // tables below follow the current lists
    qk::DevBuf<qk::MergedSeg> d_mseg;  // FP64 segments, then FP32 segments
    int m_nseg[2] = {}, m_items[2] = {}, m_grid[2] = {}, m_block = 0, m_launches = 0;
    bool m_class[qk::kNumClasses] = {};   // classes the merged launches cover
    long long last_quart = 0, last_primq = 0;
    int last_launches = 0;             // kernel launches of the last build
    int num_sms = 148;
    // device buffers
    qk::DevBuf<double> d_xyz, d_boys, d_boys8, d_D, d_cutmat, d_o;
    qk::DevBuf<int> d_q_atom, d_q_f0, d_q_parent, d_q_ltop, d_q_prim0, d_q_nprim, d_shell_f0, d_shell_f1;
    qk::DevBuf<unsigned long long> d_A, d_A2;   // d_A2: the exchange-only half of a UHF build
    qk::DevBuf<double> d_uhf;                     // UHF: Dt and Ds (2 nbasis^2), then Db and ob for host calls
    qk::DevBuf<int> d_counters;
    // optional per-class timing (CUDA events on the launching stream) and work counters
    bool profile_events = false, profile_stats = false;
    cudaEvent_t ev[2 * qk::kNumClasses] = {};
    bool ev_recorded[qk::kNumClasses] = {};
    qk::DevBuf<unsigned long long> d_stats;
    // Schwarz-bound scratch (per pair class work lists and the bit-pattern maxima)
    qk::DevBuf<unsigned long long> d_schwarz_Y, d_schwarz_cp;
    qk::DevBuf<int2> d_schwarz_work[(QK_MAX_L + 1) * (QK_MAX_L + 1)];
    // concurrent class launches: fork/join over auxiliary streams
    static constexpr int kAux = 4;
    cudaStream_t aux[kAux] = {};
    cudaEvent_t fork_ev = nullptr, join_ev[kAux] = {};
    std::vector<int> launch_order;   // class indices, coop classes first, then by listed work
    // drop-in (reference-shaped) state
    std::vector<double> host_D, host_cutmat;
    std::vector<double> host_Db;            // beta density (gpu_upload_calculated_beta_)
    bool have_D = false, have_Db = false, have_cutmat = false;
};

namespace qk {

static std::atomic<int> g_last_status{QK_OK};
static std::mutex g_default_mu;
static qk_ctx* g_default = nullptr;
static int g_default_device = 0;
static int g_maxprim_default = 20;

static int fail(int status, const char* what) {
    g_last_status = status;
    fprintf(stderr, "quick_b200: %s (status %d: %s)\n", what, status, qk_status_string(status));
    return status;
}

#define QK_CUDA_TRY(expr)                                                              \
    do {                                                                               \
        cudaError_t e_ = (expr);                                                       \
        if (e_ != cudaSuccess) {                                                       \
            fprintf(stderr, "quick_b200: CUDA error %s at %s:%d\n", cudaGetErrorString(e_), \
                    __FILE__, __LINE__);                                               \
            g_last_status = (e_ == cudaErrorMemoryAllocation) ? QK_ERR_OUT_OF_MEMORY : QK_ERR_CUDA; \
            return g_last_status.load();                                               \
        }                                                                              \
    } while (0)

static int ncart(int L) { return (L + 1) * (L + 2) / 2; }

// QUICK order of Cartesian components in a shell of momentum L (src/basis.f90:589-720)
static void cart_of(int L, int k, int out[3]) {
    int idx = 0;
    for (int nz = 0; nz <= L; ++nz)
        for (int ny = 0; ny <= L - nz; ++ny) {
            if (idx == k) { out[0] = L - nz - ny; out[1] = ny; out[2] = nz; return; }
            ++idx;
        }
}

static double cons_expected(const int c[3]) {
    int L = c[0] + c[1] + c[2];
    int nz = (c[0] > 0) + (c[1] > 0) + (c[2] > 0);
    if (L <= 1) return 1.0;
    if (L == 2) return nz == 1 ? 1.0 : std::sqrt(3.0);
    if (L == 3) {
        if (nz == 1) return 1.0;
        if (nz == 2) return std::sqrt(5.0);
        return std::sqrt(5.0) * std::sqrt(3.0);
    }
    return 1.0;
}

static DevData make_devdata(qk_ctx* c) {
    DevData d{};
    d.nbasis = c->nbasis;
    d.nshell = c->nshell;
    d.xyz = c->d_xyz.p;
    d.q_atom = c->d_q_atom.p;
    d.q_f0 = c->d_q_f0.p;
    d.q_parent = c->d_q_parent.p;
    d.q_ltop = c->d_q_ltop.p;
    d.pr_qa = c->pairs.d_qa.p;
    d.pr_qb = c->pairs.d_qb.p;
    d.pr_pp0 = c->pairs.d_pp0.p;
    d.pr_npp = c->pairs.d_npp.p;
    d.pr_pps = c->pairs.d_pps.p;
    d.pr_Y = c->pairs.d_Y.p;
    d.pr_sh = c->pairs.d_sh.p;
    d.pr_lt = c->pairs.d_lt.p;
    d.pr_geo = c->pairs.d_geo.p;
    d.pp_zo = c->pairs.d_zo.p;
    d.pp_kc = c->pairs.d_kc.p;
    d.pp_pxy = c->pairs.d_pxy.p;
    d.pp_pzax = c->pairs.d_pzax.p;
    d.pp_payz = c->pairs.d_payz.p;
    d.boys = c->d_boys.p;
    d.boys8 = (const double2*)c->d_boys8.p;
    d.cut = c->integralCutoff;
    d.primLimit = c->primLimit;
    d.boys_mode = c->boys_mode;
    return d;
}

// Canonical Qshell pairs: higher momentum first, equal momenta in index order.
// screened: keep pairs with Y * Ymax > cutoff, bucket by (La, Lb, npa, npb),
// sort each bucket by Y descending.  Otherwise keep every pair in one pass.
static void build_pairs(qk_ctx* c, bool screened) {
    PairTable& T = c->pairs;
    T.clear();
    const int nq = (int)c->qsh.size();
    struct Cand { int qa, qb; double Y; };
    std::vector<Cand> cand;
    double Ymax = 0.0;
    if (screened)
        for (double y : c->Ycut) Ymax = std::max(Ymax, y);
    for (int i = 0; i < nq; ++i)
        for (int j = 0; j < nq; ++j) {
            const Qsh &a = c->qsh[i], &b = c->qsh[j];
            if (a.L < b.L || (a.L == b.L && i > j)) continue;
            double Y = 0.0;
            if (screened) {
                Y = c->Ycut[(size_t)a.parent * c->nshell + b.parent];
                if (!(Y * Ymax > c->integralCutoff)) continue;
            }
            cand.push_back({i, j, Y});
        }
    if (screened) {
        std::stable_sort(cand.begin(), cand.end(), [&](const Cand& x, const Cand& y) {
            const Qsh &xa = c->qsh[x.qa], &xb = c->qsh[x.qb], &ya = c->qsh[y.qa], &yb = c->qsh[y.qb];
            auto kx = std::make_tuple(xa.L, xb.L, xa.nprim, xb.nprim);
            auto ky = std::make_tuple(ya.L, yb.L, ya.nprim, yb.nprim);
            if (kx != ky) return kx < ky;
            return x.Y > y.Y;
        });
    }
    for (size_t k = 0; k < cand.size(); ++k) {
        const Qsh &a = c->qsh[cand[k].qa], &b = c->qsh[cand[k].qb];
        if (screened) {
            if (T.buckets.empty() || T.buckets.back().La != a.L || T.buckets.back().Lb != b.L ||
                T.buckets.back().npa != a.nprim || T.buckets.back().npb != b.nprim)
                T.buckets.push_back({a.L, b.L, a.nprim, b.nprim, (int)k, (int)k});
            T.buckets.back().end = (int)k + 1;
        }
        T.qa.push_back(cand[k].qa);
        T.qb.push_back(cand[k].qb);
        T.Y.push_back(cand[k].Y);
        T.npp.push_back(a.nprim * b.nprim);
    }
    // primitive-pair placement: bucket-interleaved (screened) or pair-major (one
    // bucket per pair when unscreened)
    const int np = (int)cand.size();
    T.pp0.assign(np, 0);
    T.pps.assign(np, 1);
    size_t total = 0;
    if (screened) {
        for (const Bucket& B : T.buckets) {
            const int m = B.end - B.begin;
            for (int P = B.begin; P < B.end; ++P) {
                T.pp0[P] = (int)(total + (P - B.begin));
                T.pps[P] = m;
            }
            total += (size_t)m * B.npa * B.npb;
        }
    } else {
        for (int P = 0; P < np; ++P) {
            T.pp0[P] = (int)total;
            total += T.npp[P];
        }
    }
    const double2 zero2 = make_double2(0.0, 0.0);
    T.zo.assign(total, zero2); T.kc.assign(total, zero2); T.pxy.assign(total, zero2);
    T.pzax.assign(total, zero2); T.payz.assign(total, zero2);
    const double sqrtX0 = std::sqrt(kX0);
    for (int P = 0; P < np; ++P) {
        const Qsh &a = c->qsh[T.qa[P]], &b = c->qsh[T.qb[P]];
        const double* A = &c->xyz[3 * a.atom];
        const double* B = &c->xyz[3 * b.atom];
        const double r2 = (A[0] - B[0]) * (A[0] - B[0]) + (A[1] - B[1]) * (A[1] - B[1]) + (A[2] - B[2]) * (A[2] - B[2]);
        for (int i = 0; i < a.nprim; ++i)
            for (int j = 0; j < b.nprim; ++j) {
                const size_t at = (size_t)T.pp0[P] + (size_t)(i * b.nprim + j) * T.pps[P];
                const double ea = a.expo[i], eb = b.expo[j], z = ea + eb;
                // Xcoeff without X0 (src/modules/include/eri.fh:118-140)
                // Xcoeff without X0 (src/modules/include/eri.fh:118-140) times sqrt(X0): the
                // product of a bra's and a ket's K carries the whole X0
                const double K = std::exp(-ea * eb / z * r2) / z * a.coef[i] * b.coef[j] * sqrtX0;
                const double cut = screened ? c->cutprim[(size_t)(a.prim0 + i) * c->jbasis + (b.prim0 + j)] : 0.0;
                T.kc[at] = make_double2(K, cut);
                T.zo[at] = make_double2(z, 0.5 / z);
                const double px = (A[0] * ea + B[0] * eb) / z, py = (A[1] * ea + B[1] * eb) / z,
                             pz = (A[2] * ea + B[2] * eb) / z;
                T.pxy[at] = make_double2(px, py);
                T.pzax[at] = make_double2(pz, px - A[0]);
                T.payz[at] = make_double2(py - A[1], pz - A[2]);
            }
    }
}

static int upload_pairs(qk_ctx* c) {
    PairTable& T = c->pairs;
    cudaStream_t s = c->stream;
    QK_CUDA_TRY(T.d_qa.upload(T.qa, s));
    QK_CUDA_TRY(T.d_qb.upload(T.qb, s));
    QK_CUDA_TRY(T.d_pp0.upload(T.pp0, s));
    QK_CUDA_TRY(T.d_npp.upload(T.npp, s));
    QK_CUDA_TRY(T.d_pps.upload(T.pps, s));
    QK_CUDA_TRY(T.d_Y.upload(T.Y, s));
    QK_CUDA_TRY(T.d_zo.upload(T.zo, s));
    QK_CUDA_TRY(T.d_kc.upload(T.kc, s));
    QK_CUDA_TRY(T.d_pxy.upload(T.pxy, s));
    QK_CUDA_TRY(T.d_pzax.upload(T.pzax, s));
    QK_CUDA_TRY(T.d_payz.upload(T.payz, s));
    // per-pair records of DevData (pr_sh, pr_lt, pr_geo)
    const size_t np = T.qa.size();
    std::vector<int4> sh(np);
    std::vector<int> lt(np);
    std::vector<double2> geo(3 * np);
    for (size_t p = 0; p < np; ++p) {
        const Qsh& a = c->qsh[T.qa[p]];
        const Qsh& b = c->qsh[T.qb[p]];
        sh[p] = make_int4(a.parent, b.parent, a.f0, b.f0);
        lt[p] = c->q_ltop_h[T.qa[p]] + c->q_ltop_h[T.qb[p]];
        const double* A = &c->xyz[3 * a.atom];
        const double* B = &c->xyz[3 * b.atom];
        geo[3 * p] = make_double2(A[0], A[1]);
        geo[3 * p + 1] = make_double2(A[2], A[0] - B[0]);
        geo[3 * p + 2] = make_double2(A[1] - B[1], A[2] - B[2]);
    }
    QK_CUDA_TRY(T.d_sh.upload(sh, s));
    QK_CUDA_TRY(T.d_lt.upload(lt, s));
    QK_CUDA_TRY(T.d_geo.upload(geo, s));
    // the host vectors die here: the uploads must be done before they go
    QK_CUDA_TRY(cudaStreamSynchronize(s));
    return QK_OK;
}

// Work items of every class: (bra pair, first ket, count) chunks of <= 32
// kets that pass the Schwarz test, unique quartets only.
// Launch shape of class ci for the context's current work list: warps per block
// (tuned or default), the matching dynamic shared memory (cooperative classes:
// one work area per warp), and a persistent grid of as many blocks as can be
// resident (optionally capped per SM), but no more than there are items.
// Resident blocks per SM of a class kernel for a launch shape: the same for every
// context on a device, so asked once (the query costs tens of microseconds).
static cudaError_t occupancy(int device, int ci, int part, int wpb, size_t smem, int* bps) {
    static std::mutex mu;
    static std::map<std::tuple<int, int, int, int, size_t>, int> cache;
    const auto key = std::make_tuple(device, ci, part, wpb, smem);
    {
        std::lock_guard<std::mutex> g(mu);
        auto it = cache.find(key);
        if (it != cache.end()) { *bps = it->second; return cudaSuccess; }
    }
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(bps, g_classes[ci].kernel(part == 1), 32 * wpb, smem);
    if (e == cudaSuccess) {
        std::lock_guard<std::mutex> g(mu);
        cache[key] = *bps;
    }
    return e;
}

static int class_launch_shape(qk_ctx* c, int ci) {
    const ClassEntry& ce = g_classes[ci];
    ClassWork& W = c->work[ci];
    const int wpb = c->cls_wpb[ci] > 0 ? c->cls_wpb[ci] : (ce.coop ? ce.coop_warps : kWarpsPerBlock);
    const size_t smem = ce.coop ? ce.smem / ce.coop_warps * wpb : 0;
    if (smem > 48 * 1024)
        QK_CUDA_TRY(cudaFuncSetAttribute(ce.kernel(false), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ce.smem));
    for (int part = 0; part < 2; ++part) {
        const long long n = part == 0 ? W.n64 : (long long)W.n_items - W.n64;
        int& grid = part == 0 ? W.grid : W.grid32;
        grid = 0;
        if (n <= 0) continue;
        int bps = 0;
        QK_CUDA_TRY(occupancy(c->device, ci, part, wpb, smem, &bps));
        if (bps < 1) return fail(QK_ERR_CUDA, "class kernel cannot be resident");
        if (c->cls_bpsm[ci] > 0) bps = std::min(bps, c->cls_bpsm[ci]);
        grid = (int)std::max<long long>(1, std::min<long long>((long long)bps * c->num_sms, (n + wpb - 1) / wpb));
    }
    W.block = 32 * wpb;
    W.smem = smem;
    return QK_OK;
}

static int finish_work(qk_ctx* c);

// Work items of every class built on the host (the reference implementation of
// the lists; the device builder, build_work_device, gives the same lists and is
// the default except for sharded contexts).
static int build_work(qk_ctx* c) {
    PairTable& T = c->pairs;
    const double cut = c->integralCutoff;
    for (int ci = 0; ci < kNumClasses; ++ci) {
        const ClassEntry& ce = g_classes[ci];
        ClassWork& W = c->work[ci];
        W.items.clear();
        W.nquart = W.nprimq = W.nquart32 = 0;
        const bool same = (ce.La == ce.Lc && ce.Lb == ce.Ld);
        struct Tmp { int4 it; long long cost; };
        std::vector<Tmp> tmp;
        for (int bb = 0; bb < (int)T.buckets.size(); ++bb) {
            const Bucket& B = T.buckets[bb];
            if (B.La != ce.La || B.Lb != ce.Lb) continue;
            for (int kb = 0; kb < (int)T.buckets.size(); ++kb) {
                const Bucket& K = T.buckets[kb];
                if (K.La != ce.Lc || K.Lb != ce.Ld) continue;
                if (same && kb > bb) continue;
                const long long cost = (long long)B.npa * B.npb * K.npa * K.npb;
                for (int P = B.begin; P < B.end; ++P) {
                    const double yp = T.Y[P];
                    // prefix of the ket bucket with yp * yq > cut (Y sorted descending)
                    int lo = K.begin, hi = K.end;
                    while (lo < hi) {
                        int mid = (lo + hi) / 2;
                        if (yp * T.Y[mid] > cut) lo = mid + 1; else hi = mid;
                    }
                    int nk = lo - K.begin;
                    if (same && kb == bb) nk = std::min(nk, P - B.begin + 1);
                    if (nk <= 0) continue;
                    W.nquart += nk;
                    W.nprimq += (long long)T.npp[P] * K.npa * K.npb * nk;
                    // per-lane classes: up to 32 kets per warp item; cooperative classes
                    // (one quartet per warp at a time): one ket per item, so that the
                    // few, long quartets spread over many warps
                    const int chunk = ce.coop ? 1 : 32;
                    // mixed form: kets with yp * yq below fp32_bound (a suffix, Y sorted
                    // descending) go to FP32 items; the cooperative classes stay FP64
                    int n64 = nk;
                    if (c->fp32_bound > 0.0 && !ce.coop) {
                        int a = 0, z = nk;
                        while (a < z) {
                            const int mid = (a + z) / 2;
                            if (yp * T.Y[K.begin + mid] >= c->fp32_bound) a = mid + 1; else z = mid;
                        }
                        n64 = a;
                    }
                    W.nquart32 += nk - n64;
                    for (int s = 0; s < n64; s += chunk)
                        tmp.push_back({make_int4(P, K.begin + s, std::min(chunk, n64 - s), 0), cost});
                    for (int s = n64; s < nk; s += chunk)
                        tmp.push_back({make_int4(P, K.begin + s, std::min(chunk, nk - s), 1), cost});
                }
            }
        }
        // FP64 items first, then the FP32 ones (two launches); each part by cost
        std::stable_sort(tmp.begin(), tmp.end(), [](const Tmp& x, const Tmp& y) {
            if (x.it.w != y.it.w) return x.it.w < y.it.w;
            return x.cost > y.cost;
        });
        // a shard keeps every shard_count-th item of the cost-ordered list (each
        // precision part stays cost-ordered), so the shards' work is balanced
        if (c->shard_count > 1) {
            size_t k = 0;
            for (size_t i = 0; i < tmp.size(); ++i)
                if ((int)(i % (size_t)c->shard_count) == c->shard_rank) tmp[k++] = tmp[i];
            tmp.resize(k);
            W.nquart = W.nprimq = W.nquart32 = 0;
            for (const Tmp& t : tmp) {
                W.nquart += t.it.z;
                W.nprimq += t.cost * t.it.z;
                if (t.it.w == 1) W.nquart32 += t.it.z;
            }
        }
        W.n64 = 0;
        for (const Tmp& t : tmp) W.n64 += t.it.w == 0;
        W.items.resize(tmp.size());
        for (size_t i = 0; i < tmp.size(); ++i) W.items[i] = tmp[i].it;
        W.n_items = (int)W.items.size();
    }
    // one device buffer for every class's items, class after class
    std::vector<int4> all;
    std::vector<size_t> first(kNumClasses);
    for (int ci = 0; ci < kNumClasses; ++ci) {
        first[ci] = all.size();
        all.insert(all.end(), c->work[ci].items.begin(), c->work[ci].items.end());
    }
    QK_CUDA_TRY(c->d_items.upload(all, c->stream));
    for (int ci = 0; ci < kNumClasses; ++ci) c->work[ci].d_items = c->d_items.p + first[ci];
    return finish_work(c);
}

// Launch shapes, launch count and launch order of the work lists just built.
static int finish_work(qk_ctx* c) {
    c->launches = 0;
    for (int ci = 0; ci < kNumClasses; ++ci) {
        ClassWork& W = c->work[ci];
        if (W.n_items > 0) {
            int st = class_launch_shape(c, ci);
            if (st) return st;
            c->launches += (W.n64 > 0) + (W.n64 < W.n_items);
        }
    }
    c->launches += 1;  // finalize
    c->launch_order.clear();
    for (int ci = 0; ci < kNumClasses; ++ci)
        if (c->work[ci].n_items > 0) c->launch_order.push_back(ci);
    std::stable_sort(c->launch_order.begin(), c->launch_order.end(), [&](int x, int y) {
        if (g_classes[x].coop != g_classes[y].coop) return g_classes[x].coop;
        const double wx = c->work[x].nprimq * g_classes[x].prim_flops + c->work[x].nquart * g_classes[x].quartet_flops;
        const double wy = c->work[y].nprimq * g_classes[y].prim_flops + c->work[y].nquart * g_classes[y].quartet_flops;
        return wx > wy;
    });
    if (!c->fork_ev) {
        QK_CUDA_TRY(cudaEventCreateWithFlags(&c->fork_ev, cudaEventDisableTiming));
        for (int k = 0; k < qk_ctx::kAux; ++k) {
            QK_CUDA_TRY(cudaStreamCreateWithFlags(&c->aux[k], cudaStreamNonBlocking));
            QK_CUDA_TRY(cudaEventCreateWithFlags(&c->join_ev[k], cudaEventDisableTiming));
        }
    }
    return QK_OK;
}

// ------------------------------------------------------------------ work lists on the device
// The same lists as build_work, built by the GPU: a segment is one (bra bucket,
// ket bucket) pair of a class, and one thread per (segment, bra pair) finds its
// ket prefix by binary search (wl_count_kernel); exclusive scans of the FP64 and
// FP32 item counts give every thread its place (wl_emit_kernel).  The segments of
// a class are ordered by cost on the host exactly as build_work's stable sort
// orders the items, so the lists are identical item for item.
struct WlSeg {
    int bra0, bra1;        // bra pairs [bra0, bra1)
    int ket0, ket1;        // ket bucket [ket0, ket1), Y descending
    int ci;                // class
    int chunk;             // kets per item: 32 (per-lane classes) or 1 (cooperative)
    int tri;               // bra and ket bucket are the same: kets Q <= P only
    int fp32_ok;           // the mixed form may put this segment's small-bound kets in FP32 items
    long long ket_npp;     // primitive pairs of one ket pair
    int t0;                // first thread of the segment
    int pad;
};

__device__ __forceinline__ int wl_find_seg(const WlSeg* __restrict__ segs, int nseg, int t) {
    int lo = 0, hi = nseg - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (segs[mid].t0 <= t) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__global__ void wl_count_kernel(const WlSeg* __restrict__ segs, int nseg, int nthreads, const double* __restrict__ Y,
                                const int* __restrict__ npp, double cut, double fp32_bound, int* __restrict__ nk_out,
                                int* __restrict__ n64_out, int* __restrict__ c64, int* __restrict__ c32,
                                unsigned long long* __restrict__ stats) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nthreads) return;
    const WlSeg sg = segs[wl_find_seg(segs, nseg, t)];
    const int P = sg.bra0 + (t - sg.t0);
    const double yp = Y[P];
    int lo = sg.ket0, hi = sg.ket1;
    while (lo < hi) {
        const int mid = (lo + hi) / 2;
        if (yp * Y[mid] > cut) lo = mid + 1; else hi = mid;
    }
    int nk = lo - sg.ket0;
    if (sg.tri) nk = min(nk, P - sg.bra0 + 1);
    int n64 = nk;
    if (nk > 0 && fp32_bound > 0.0 && sg.fp32_ok) {
        int a = 0, z = nk;
        while (a < z) {
            const int mid = (a + z) / 2;
            if (yp * Y[sg.ket0 + mid] >= fp32_bound) a = mid + 1; else z = mid;
        }
        n64 = a;
    }
    if (nk < 0) nk = 0;
    nk_out[t] = nk;
    n64_out[t] = n64;
    c64[t] = nk > 0 ? (n64 + sg.chunk - 1) / sg.chunk : 0;
    c32[t] = nk > 0 ? (nk - n64 + sg.chunk - 1) / sg.chunk : 0;
    if (nk > 0) {
        atomicAdd(stats + 3 * sg.ci, (unsigned long long)nk);
        atomicAdd(stats + 3 * sg.ci + 1, (unsigned long long)npp[P] * (unsigned long long)sg.ket_npp * nk);
        atomicAdd(stats + 3 * sg.ci + 2, (unsigned long long)(nk - n64));
    }
}

// per class: FP64 and FP32 item totals from the scans (threads [t0, t1) of the class)
__global__ void wl_totals_kernel(const int* __restrict__ ct0, const int* __restrict__ ct1, const int* __restrict__ c64,
                                 const int* __restrict__ off64, const int* __restrict__ c32,
                                 const int* __restrict__ off32, int ncls, int* __restrict__ tot) {
    const int ci = threadIdx.x;
    if (ci >= ncls) return;
    const int a = ct0[ci], b = ct1[ci];
    tot[2 * ci] = b > a ? off64[b - 1] + c64[b - 1] - off64[a] : 0;
    tot[2 * ci + 1] = b > a ? off32[b - 1] + c32[b - 1] - off32[a] : 0;
}

// cls: per class [first thread, item base, FP64 items]
__global__ void wl_emit_kernel(const WlSeg* __restrict__ segs, int nseg, int nthreads, const int* __restrict__ nk_in,
                               const int* __restrict__ n64_in, const int* __restrict__ off64,
                               const int* __restrict__ off32, const int* __restrict__ cls, int4* __restrict__ items) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nthreads) return;
    const int nk = nk_in[t];
    if (nk <= 0) return;
    const WlSeg sg = segs[wl_find_seg(segs, nseg, t)];
    const int P = sg.bra0 + (t - sg.t0);
    const int n64 = n64_in[t];
    const int first = cls[3 * sg.ci], base = cls[3 * sg.ci + 1], n64c = cls[3 * sg.ci + 2];
    int4* o = items + base + (off64[t] - off64[first]);
    for (int k = 0; k < n64; k += sg.chunk) *o++ = make_int4(P, sg.ket0 + k, min(sg.chunk, n64 - k), 0);
    o = items + base + n64c + (off32[t] - off32[first]);
    for (int k = n64; k < nk; k += sg.chunk) *o++ = make_int4(P, sg.ket0 + k, min(sg.chunk, nk - k), 1);
}

static size_t wl_align(size_t x) { return (x + 255) & ~(size_t)255; }

// build_work on the GPU (pair tables already uploaded on the context stream); two
// small host synchronisations: the class totals, and the end of prepare.
static int build_work_device(qk_ctx* c) {
    PairTable& T = c->pairs;
    cudaStream_t s = c->stream;
    // segments, class by class, each class's in build_work's item order
    std::vector<WlSeg> segs;
    std::vector<int> ct0(kNumClasses), ct1(kNumClasses);
    int nthreads = 0;
    for (int ci = 0; ci < kNumClasses; ++ci) {
        const ClassEntry& ce = g_classes[ci];
        const bool same = (ce.La == ce.Lc && ce.Lb == ce.Ld);
        struct Cand { WlSeg sg; long long cost; };
        std::vector<Cand> cand;
        for (int bb = 0; bb < (int)T.buckets.size(); ++bb) {
            const Bucket& B = T.buckets[bb];
            if (B.La != ce.La || B.Lb != ce.Lb) continue;
            for (int kb = 0; kb < (int)T.buckets.size(); ++kb) {
                const Bucket& K = T.buckets[kb];
                if (K.La != ce.Lc || K.Lb != ce.Ld) continue;
                if (same && kb > bb) continue;
                WlSeg sg{};
                sg.bra0 = B.begin; sg.bra1 = B.end; sg.ket0 = K.begin; sg.ket1 = K.end;
                sg.ci = ci; sg.chunk = ce.coop ? 1 : 32; sg.tri = (same && kb == bb) ? 1 : 0;
                sg.fp32_ok = ce.coop ? 0 : 1;
                sg.ket_npp = (long long)K.npa * K.npb;
                cand.push_back({sg, (long long)B.npa * B.npb * K.npa * K.npb});
            }
        }
        std::stable_sort(cand.begin(), cand.end(), [](const Cand& x, const Cand& y) { return x.cost > y.cost; });
        ct0[ci] = nthreads;
        for (auto& cd : cand) {
            cd.sg.t0 = nthreads;
            nthreads += cd.sg.bra1 - cd.sg.bra0;
            segs.push_back(cd.sg);
        }
        ct1[ci] = nthreads;
    }
    for (int ci = 0; ci < kNumClasses; ++ci) {
        ClassWork& W = c->work[ci];
        W.items.clear();
        W.nquart = W.nprimq = W.nquart32 = 0;
        W.n64 = W.n_items = 0;
        W.d_items = nullptr;
    }
    if (nthreads == 0) return finish_work(c);
    const int nseg = (int)segs.size();
    // scratch layout
    size_t cub_bytes = 0;
    QK_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, cub_bytes, (int*)nullptr, (int*)nullptr, nthreads, s));
    const size_t nt = (size_t)nthreads;
    size_t off = 0;
    const size_t o_seg = off; off = wl_align(off + sizeof(WlSeg) * nseg);
    const size_t o_nk = off; off = wl_align(off + 4 * nt);
    const size_t o_n64 = off; off = wl_align(off + 4 * nt);
    const size_t o_c64 = off; off = wl_align(off + 4 * nt);
    const size_t o_c32 = off; off = wl_align(off + 4 * nt);
    const size_t o_off64 = off; off = wl_align(off + 4 * nt);
    const size_t o_off32 = off; off = wl_align(off + 4 * nt);
    const size_t o_stats = off; off = wl_align(off + 8 * 3 * kNumClasses);
    const size_t o_ct = off; off = wl_align(off + 4 * 2 * kNumClasses);
    const size_t o_tot = off; off = wl_align(off + 4 * 2 * kNumClasses);
    const size_t o_cls = off; off = wl_align(off + 4 * 3 * kNumClasses);
    const size_t o_cub = off; off = wl_align(off + cub_bytes);
    QK_CUDA_TRY(c->d_wl.reserve(off));
    char* w = c->d_wl.p;
    WlSeg* d_seg = (WlSeg*)(w + o_seg);
    int *d_nk = (int*)(w + o_nk), *d_n64 = (int*)(w + o_n64), *d_c64 = (int*)(w + o_c64), *d_c32 = (int*)(w + o_c32);
    int *d_off64 = (int*)(w + o_off64), *d_off32 = (int*)(w + o_off32);
    unsigned long long* d_stats = (unsigned long long*)(w + o_stats);
    int *d_ct = (int*)(w + o_ct), *d_tot = (int*)(w + o_tot), *d_cls = (int*)(w + o_cls);
    std::vector<int> ct(2 * kNumClasses);
    for (int ci = 0; ci < kNumClasses; ++ci) { ct[ci] = ct0[ci]; ct[kNumClasses + ci] = ct1[ci]; }
    QK_CUDA_TRY(cudaMemcpyAsync(d_seg, segs.data(), sizeof(WlSeg) * nseg, cudaMemcpyHostToDevice, s));
    QK_CUDA_TRY(cudaMemcpyAsync(d_ct, ct.data(), sizeof(int) * 2 * kNumClasses, cudaMemcpyHostToDevice, s));
    QK_CUDA_TRY(cudaMemsetAsync(d_stats, 0, 8 * 3 * kNumClasses, s));
    const int nb = (nthreads + 255) / 256;
    wl_count_kernel<<<nb, 256, 0, s>>>(d_seg, nseg, nthreads, T.d_Y.p, T.d_npp.p, c->integralCutoff, c->fp32_bound,
                                       d_nk, d_n64, d_c64, d_c32, d_stats);
    QK_CUDA_TRY(cudaGetLastError());
    size_t tb = cub_bytes;
    QK_CUDA_TRY(cub::DeviceScan::ExclusiveSum(w + o_cub, tb, d_c64, d_off64, nthreads, s));
    tb = cub_bytes;
    QK_CUDA_TRY(cub::DeviceScan::ExclusiveSum(w + o_cub, tb, d_c32, d_off32, nthreads, s));
    wl_totals_kernel<<<1, 64, 0, s>>>(d_ct, d_ct + kNumClasses, d_c64, d_off64, d_c32, d_off32, kNumClasses, d_tot);
    QK_CUDA_TRY(cudaGetLastError());
    std::vector<int> tot(2 * kNumClasses);
    std::vector<unsigned long long> st(3 * kNumClasses);
    QK_CUDA_TRY(cudaMemcpyAsync(tot.data(), d_tot, sizeof(int) * 2 * kNumClasses, cudaMemcpyDeviceToHost, s));
    QK_CUDA_TRY(cudaMemcpyAsync(st.data(), d_stats, 8 * 3 * kNumClasses, cudaMemcpyDeviceToHost, s));
    QK_CUDA_TRY(cudaStreamSynchronize(s));
    std::vector<int> cls(3 * kNumClasses);
    long long total = 0;
    for (int ci = 0; ci < kNumClasses; ++ci) {
        ClassWork& W = c->work[ci];
        W.n64 = tot[2 * ci];
        W.n_items = tot[2 * ci] + tot[2 * ci + 1];
        W.nquart = (long long)st[3 * ci];
        W.nprimq = (long long)st[3 * ci + 1];
        W.nquart32 = (long long)st[3 * ci + 2];
        cls[3 * ci] = ct0[ci];
        cls[3 * ci + 1] = (int)total;
        cls[3 * ci + 2] = W.n64;
        total += W.n_items;
    }
    if (total > INT_MAX) return fail(QK_ERR_UNSUPPORTED, "more than 2^31 work items");
    QK_CUDA_TRY(c->d_items.reserve((size_t)std::max<long long>(total, 1)));
    QK_CUDA_TRY(cudaMemcpyAsync(d_cls, cls.data(), sizeof(int) * 3 * kNumClasses, cudaMemcpyHostToDevice, s));
    wl_emit_kernel<<<nb, 256, 0, s>>>(d_seg, nseg, nthreads, d_nk, d_n64, d_off64, d_off32, d_cls, c->d_items.p);
    QK_CUDA_TRY(cudaGetLastError());
    for (int ci = 0; ci < kNumClasses; ++ci) c->work[ci].d_items = c->d_items.p + cls[3 * ci + 1];
    return finish_work(c);
}

static int ensure_pairs(qk_ctx* c) {
    if (!c->have_basis) return fail(QK_ERR_NOT_READY, "basis not uploaded");
    if (!c->have_schwarz) return fail(QK_ERR_NOT_READY, "Schwarz bounds not set");
    // Lists built at a tighter cutoff than the one in force are kept: they hold
    // every quartet the looser cutoff admits, and the kernels apply the cutoff in
    // force themselves (an SCF that tightens its cutoff as it converges builds
    // its lists once, at the final cutoff).
    if (!c->pairs_dirty && c->built_cut <= c->integralCutoff && c->built_fp32 == c->fp32_bound) return QK_OK;
    build_pairs(c, true);
    int st = upload_pairs(c);
    if (st) return st;
    // the device builder, except for sharded contexts (the host one deals items to shards)
    st = (c->worklist_on_device && c->shard_count == 1) ? build_work_device(c) : build_work(c);
    if (st) return st;
    // tables were uploaded on the context stream; builds may run on another stream
    QK_CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->built_cut = c->integralCutoff;
    c->built_fp32 = c->fp32_bound;
    c->pairs_dirty = false;
    c->m_ready = false;
    return QK_OK;
}

// The segment tables and launch shapes of the merged s/p launches for the current
// lists (qk_set_merge_sp); m_launches = the build's launches with them.
static int prepare_merged(qk_ctx* c) {
#if QK_MAX_L >= 1
    std::vector<MergedSeg> segs[2];
    int total[2] = {0, 0};
    for (int k = 0; k < kNumClasses; ++k) c->m_class[k] = false;
    int replaced = 0;
    for (int m = 0; m < kSpMergedN; ++m) {
        int ci = -1;
        for (int k = 0; k < kNumClasses; ++k)
            if (g_classes[k].La == kSpMerged[m][0] && g_classes[k].Lb == kSpMerged[m][1] &&
                g_classes[k].Lc == kSpMerged[m][2] && g_classes[k].Ld == kSpMerged[m][3] && !g_classes[k].coop)
                ci = k;
        if (ci < 0) continue;
        const ClassWork& W = c->work[ci];
        c->m_class[ci] = true;
        replaced += (W.n64 > 0) + (W.n64 < W.n_items);
        const int n[2] = {W.n64, W.n_items - W.n64};
        const int4* it[2] = {W.d_items, W.d_items + W.n64};
        for (int part = 0; part < 2; ++part)
            if (n[part] > 0) {
                segs[part].push_back({it[part], total[part], m});
                total[part] += n[part];
            }
    }
    std::vector<MergedSeg> all(segs[0]);
    all.insert(all.end(), segs[1].begin(), segs[1].end());
    if (!all.empty()) {
        QK_CUDA_TRY(c->d_mseg.upload(all, c->stream));
        QK_CUDA_TRY(cudaStreamSynchronize(c->stream));
    }
    const int wpb = kWarpsPerBlock;
    c->m_block = 32 * wpb;
    int parts = 0;
    for (int part = 0; part < 2; ++part) {
        c->m_nseg[part] = (int)segs[part].size();
        c->m_items[part] = total[part];
        c->m_grid[part] = 0;
        if (total[part] == 0) continue;
        int bps = 0;
        const void* fn = part ? (const void*)fock_merged_sp_kernel<true> : (const void*)fock_merged_sp_kernel<false>;
        QK_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, fn, c->m_block, 0));
        if (bps < 1) return fail(QK_ERR_CUDA, "merged s/p kernel cannot be resident");
        c->m_grid[part] = (int)std::max<long long>(1, std::min<long long>((long long)bps * c->num_sms,
                                                                          (total[part] + wpb - 1) / wpb));
        ++parts;
    }
    c->m_launches = c->launches - replaced + parts;
#else
    for (int k = 0; k < kNumClasses; ++k) c->m_class[k] = false;
    c->m_nseg[0] = c->m_nseg[1] = c->m_items[0] = c->m_items[1] = 0;
    c->m_launches = c->launches;
#endif
    c->m_ready = true;
    return QK_OK;
}

// One class's launches: its FP64 items, then (mixed form) its FP32 items, each
// part with its own counter (counters[ci] and counters[kNumClasses + ci]).
static void launch_class(const ClassEntry& ce, const ClassWork& W, cudaStream_t s, const DevData& d, int* counters,
                         int ci) {
    const int n = W.n_items;
    if (W.n64 > 0)
        ce.fn(false, dim3(W.grid), dim3(W.block), W.smem, s, d, W.d_items, W.n64, counters + ci);
    if (n > W.n64)
        ce.fn(true, dim3(W.grid32), dim3(W.block), W.smem, s, d, W.d_items + W.n64, n - W.n64,
              counters + kNumClasses + ci);
}

// A_ext: the caller's int64 accumulator (nbasis^2, not cleared, not finalised)
// instead of the context's, for sharded builds whose accumulators are summed
// across GPUs before the one finalisation; o is then unused.
static int fock2e_device(qk_ctx* c, const double* D, const double* cutmat, double* o, cudaStream_t s,
                         unsigned long long* A_ext = nullptr, int exchange_only = 0) {
    // a sharded context holds only its share of the work: finalising that share
    // into o would be a silently partial Fock matrix
    if (!A_ext && c->shard_count > 1)
        return fail(QK_ERR_INVALID_ARG, "context is sharded (qk_set_shard): use qk_fock2e_device_accumulate");
    int st = ensure_pairs(c);
    if (st) return st;
    const int n = c->nbasis, ns = c->nshell;
    if (!cutmat) {
        QK_CUDA_TRY(c->d_cutmat.reserve((size_t)ns * ns));
        density_cutoff_kernel<<<(ns * ns + 127) / 128, 128, 0, s>>>(D, n, ns, c->d_shell_f0.p,
                                                                     c->d_shell_f1.p, c->d_cutmat.p);
        QK_CUDA_TRY(cudaGetLastError());
        cutmat = c->d_cutmat.p;
    }
    // merged s/p launches: not when every class is timed or counted on its own
    const bool merged = c->merge_sp && !c->profile_events && !c->profile_stats;
    if (merged && !c->m_ready) {
        st = prepare_merged(c);
        if (st) return st;
    }
    QK_CUDA_TRY(c->d_counters.reserve(2 * kNumClasses + 2));
    if (!A_ext) {
        QK_CUDA_TRY(c->d_A.reserve((size_t)n * n));
        QK_CUDA_TRY(cudaMemsetAsync(c->d_A.p, 0, sizeof(unsigned long long) * n * n, s));
    }
    QK_CUDA_TRY(cudaMemsetAsync(c->d_counters.p, 0, sizeof(int) * (2 * kNumClasses + 2), s));
    DevData d = make_devdata(c);
    d.D = D;
    d.cutmat = cutmat;
    d.A = A_ext ? A_ext : c->d_A.p;
    d.stats = nullptr;
    d.exchange_only = exchange_only;
    if (c->profile_stats) {
        QK_CUDA_TRY(c->d_stats.reserve(2 * kNumClasses));
        QK_CUDA_TRY(cudaMemsetAsync(c->d_stats.p, 0, sizeof(unsigned long long) * 2 * kNumClasses, s));
    }
    long long nq = 0, npq = 0;
    for (int ci = 0; ci < kNumClasses; ++ci) c->ev_recorded[ci] = false;
    // Classes run concurrently on auxiliary streams forked from `s` (the high
    // angular momentum, latency-bound classes first so the bulk classes fill the
    // remaining SMs).  With per-class event timing on they run one after another
    // on `s`, so that every class kernel is timed alone.
    const bool concurrent = !c->profile_events && c->nstreams > 0;
#if QK_MAX_L >= 1
    if (merged) {
        // the joined s/p lists first, on the caller's stream
        for (int part = 0; part < 2; ++part)
            if (c->m_items[part] > 0) {
                const MergedSeg* sg = c->d_mseg.p + (part ? c->m_nseg[0] : 0);
                int* ctr = c->d_counters.p + 2 * kNumClasses + part;
                if (part)
                    fock_merged_sp_kernel<true><<<c->m_grid[1], c->m_block, 0, s>>>(d, sg, c->m_nseg[1],
                                                                                  c->m_items[1], ctr);
                else
                    fock_merged_sp_kernel<false><<<c->m_grid[0], c->m_block, 0, s>>>(d, sg, c->m_nseg[0],
                                                                                   c->m_items[0], ctr);
                QK_CUDA_TRY(cudaGetLastError());
            }
    }
#endif
    if (concurrent) QK_CUDA_TRY(cudaEventRecord(c->fork_ev, s));
    bool used[qk_ctx::kAux] = {};
    int slot = 0;
    for (int ci : c->launch_order) {
        ClassWork& W = c->work[ci];
        if (merged && c->m_class[ci]) {
            nq += W.nquart;
            npq += W.nprimq;
            continue;
        }
        cudaStream_t ls = s;
        if (concurrent) {
            const int k = slot++ % c->nstreams;
            ls = c->aux[k];
            if (!used[k]) {
                QK_CUDA_TRY(cudaStreamWaitEvent(ls, c->fork_ev, 0));
                used[k] = true;
            }
        }
        if (c->profile_stats) d.stats = c->d_stats.p + 2 * ci;
        if (c->profile_events) QK_CUDA_TRY(cudaEventRecord(c->ev[2 * ci], ls));
        const ClassEntry& ce = g_classes[ci];
        launch_class(ce, W, ls, d, c->d_counters.p, ci);
        QK_CUDA_TRY(cudaGetLastError());
        if (c->profile_events) {
            QK_CUDA_TRY(cudaEventRecord(c->ev[2 * ci + 1], ls));
            c->ev_recorded[ci] = true;
        }
        nq += W.nquart;
        npq += W.nprimq;
    }
    if (concurrent)
        for (int k = 0; k < qk_ctx::kAux; ++k)
            if (used[k]) {
                QK_CUDA_TRY(cudaEventRecord(c->join_ev[k], c->aux[k]));
                QK_CUDA_TRY(cudaStreamWaitEvent(s, c->join_ev[k], 0));
            }
    if (!A_ext) {
        finalize_kernel<<<(n * n + 255) / 256, 256, 0, s>>>(c->d_A.p, n, o);
        QK_CUDA_TRY(cudaGetLastError());
    }
    c->last_quart = nq;
    c->last_primq = npq;
    c->last_launches = merged ? c->m_launches : c->launches;
    return QK_OK;
}


// Open-shell (UHF) Fock build: oa += G_a, ob += G_b with G_a = J[Da + Db] - K[Da],
// G_b = J[Da + Db] - K[Db] (QUICK's get_oshell_eri, src/modules/include/eri.fh under
// OSHELL; src/gpu/gpu_get2e_subs.h:638-660).  Written as one closed-shell build of the
// total density Dt = Da + Db (J - K/2) and one exchange-only build of the spin density
// Ds = Da - Db (-K/2): G_a = G(Dt) + K(Ds), G_b = G(Dt) - K(Ds).  Both builds use the
// open-shell density screen, so their quartets are QUICK's open-shell set.
static int fock2e_uhf_device(qk_ctx* c, const double* Da, const double* Db, const double* cutmat, double* oa,
                             double* ob, cudaStream_t s) {
    if (c->shard_count > 1)
        return fail(QK_ERR_INVALID_ARG, "context is sharded (qk_set_shard): UHF builds are not sharded");
    int st = ensure_pairs(c);
    if (st) return st;
    const int n = c->nbasis, ns = c->nshell;
    const size_t nn = (size_t)n * n;
    QK_CUDA_TRY(c->d_uhf.reserve(2 * nn));
    double* Dt = c->d_uhf.p;
    double* Ds = c->d_uhf.p + nn;
    uhf_densities_kernel<<<(int)std::min<size_t>((nn + 255) / 256, 8192), 256, 0, s>>>(Da, Db, (long long)nn, Dt, Ds);
    QK_CUDA_TRY(cudaGetLastError());
    if (!cutmat) {
        QK_CUDA_TRY(c->d_cutmat.reserve((size_t)ns * ns));
        density_cutoff_uhf_kernel<<<(ns * ns + 127) / 128, 128, 0, s>>>(Da, Db, n, ns, c->d_shell_f0.p,
                                                                        c->d_shell_f1.p, c->d_cutmat.p);
        QK_CUDA_TRY(cudaGetLastError());
        cutmat = c->d_cutmat.p;
    }
    QK_CUDA_TRY(c->d_A.reserve(nn));
    QK_CUDA_TRY(c->d_A2.reserve(nn));
    QK_CUDA_TRY(cudaMemsetAsync(c->d_A.p, 0, sizeof(unsigned long long) * nn, s));
    QK_CUDA_TRY(cudaMemsetAsync(c->d_A2.p, 0, sizeof(unsigned long long) * nn, s));
    st = fock2e_device(c, Dt, cutmat, nullptr, s, c->d_A.p, 0);
    if (st) return st;
    st = fock2e_device(c, Ds, cutmat, nullptr, s, c->d_A2.p, 1);
    if (st) return st;
    finalize_uhf_kernel<<<(int)((nn + 255) / 256), 256, 0, s>>>(c->d_A.p, c->d_A2.p, n, oa, ob);
    QK_CUDA_TRY(cudaGetLastError());
    return QK_OK;
}

// ------------------------------------------------------------------ fixed scratch
// Scratch of the allocation-free build (qk_fock2e_device_noalloc).  Some callers
// may not allocate device memory at the point where they need a Fock build (a
// host program whose memory pool is fixed after start-up, a section that must
// not call cudaMalloc/cudaFree because those synchronise the device, or a
// runtime that hands this library only the buffers it owns).  For them the
// per-build scratch -- the int64 accumulator, the work counters and, when the
// caller passes no density screen, that screen -- lives in this file-scope
// array, which every GPU that loads the library holds until the process exits.
// Layout in 8-byte words: [A: kNoAllocMaxNbasis^2][cutmat: kNoAllocMaxNshell^2]
// [counters: 2 * kNumClasses ints].
constexpr int kNoAllocMaxNbasis = 1024;
constexpr int kNoAllocMaxNshell = 512;
constexpr size_t kNoAllocWordsA = (size_t)kNoAllocMaxNbasis * kNoAllocMaxNbasis;
constexpr size_t kNoAllocWordsCut = (size_t)kNoAllocMaxNshell * kNoAllocMaxNshell;
constexpr size_t kNoAllocWords = kNoAllocWordsA + kNoAllocWordsCut + kNumClasses + 1;
static __device__ __align__(256) unsigned long long g_noalloc_scratch[kNoAllocWords];

// Device address of g_noalloc_scratch, looked up once per device (in host code the
// symbol's name is only a stand-in for the device array, never a usable pointer).
constexpr int kNoAllocMaxDevices = 64;
static std::mutex g_noalloc_mu;
static unsigned long long* g_noalloc_ptr[kNoAllocMaxDevices] = {};

static int noalloc_scratch(int device, unsigned long long** out) {
    if (device < 0 || device >= kNoAllocMaxDevices) return fail(QK_ERR_UNSUPPORTED, "device index too large");
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    if (!g_noalloc_ptr[device]) {
        void* p = nullptr;
        // the caller made `device` current
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            fprintf(stderr, "quick_b200: cudaGetSymbolAddress(scratch) failed: %s\n", cudaGetErrorString(e));
            g_last_status = QK_ERR_CUDA;
            return QK_ERR_CUDA;
        }
        g_noalloc_ptr[device] = (unsigned long long*)p;
    }
    *out = g_noalloc_ptr[device];
    return QK_OK;
}

// The same build as fock2e_device with its scratch taken from g_noalloc_scratch;
// it calls no allocator.  The pair tables and work lists must already exist.
static int fock2e_device_noalloc(qk_ctx* c, const double* D, const double* cutmat, double* o, cudaStream_t s) {
    if (c->shard_count > 1)
        return fail(QK_ERR_INVALID_ARG, "context is sharded (qk_set_shard): use qk_fock2e_device_accumulate");
    if (c->nbasis > kNoAllocMaxNbasis)
        return fail(QK_ERR_INVALID_ARG, "qk_fock2e_device_noalloc: nbasis exceeds the fixed scratch (max 1024)");
    if (!cutmat && c->nshell > kNoAllocMaxNshell)
        return fail(QK_ERR_INVALID_ARG,
                    "qk_fock2e_device_noalloc: nshell exceeds the fixed density-screen scratch (max 512); "
                    "pass cutmat_dev");
    // the same test as ensure_pairs: anything that would make qk_fock2e_device rebuild
    // its lists (basis, Schwarz bounds, shard, a tighter cutoff, another FP32 bound)
    // is a refusal here, since building them allocates
    if (!c->have_basis || !c->have_schwarz || c->pairs_dirty || c->built_cut > c->integralCutoff ||
        c->built_fp32 != c->fp32_bound)
        return fail(QK_ERR_NOT_READY,
                    "qk_fock2e_device_noalloc: pair tables not built for the current basis/Schwarz/cutoffs/"
                    "precision; run qk_fock2e_device (or qk_prepare) once first");
    unsigned long long* base = nullptr;
    int st = noalloc_scratch(c->device, &base);
    if (st) return st;
    unsigned long long* A = base;
    double* cut_scratch = (double*)(base + kNoAllocWordsA);
    int* counters = (int*)(base + kNoAllocWordsA + kNoAllocWordsCut);
    const int n = c->nbasis, ns = c->nshell;
    if (!cutmat) {
        density_cutoff_kernel<<<(ns * ns + 127) / 128, 128, 0, s>>>(D, n, ns, c->d_shell_f0.p,
                                                                     c->d_shell_f1.p, cut_scratch);
        QK_CUDA_TRY(cudaGetLastError());
        cutmat = cut_scratch;
    }
    // the array keeps the previous call's contents: clear what must start at zero
    QK_CUDA_TRY(cudaMemsetAsync(A, 0, sizeof(unsigned long long) * n * n, s));
    QK_CUDA_TRY(cudaMemsetAsync(counters, 0, sizeof(int) * 2 * kNumClasses, s));
    DevData d = make_devdata(c);
    d.D = D;
    d.cutmat = cutmat;
    d.A = A;
    d.stats = nullptr;
    // the launch shape of fock2e_device: concurrent over the context's nstreams
    // auxiliary streams, or one class after another on `s` (nstreams 0)
    const bool concurrent = c->nstreams > 0;
    if (concurrent) QK_CUDA_TRY(cudaEventRecord(c->fork_ev, s));
    bool used[qk_ctx::kAux] = {};
    int slot = 0;
    long long nq = 0, npq = 0;
    for (int ci : c->launch_order) {
        const ClassWork& W = c->work[ci];
        cudaStream_t ls = s;
        if (concurrent) {
            const int k = slot++ % c->nstreams;
            ls = c->aux[k];
            if (!used[k]) {
                QK_CUDA_TRY(cudaStreamWaitEvent(ls, c->fork_ev, 0));
                used[k] = true;
            }
        }
        const ClassEntry& ce = g_classes[ci];
        launch_class(ce, W, ls, d, counters, ci);
        QK_CUDA_TRY(cudaGetLastError());
        nq += W.nquart;
        npq += W.nprimq;
    }
    if (concurrent)
        for (int k = 0; k < qk_ctx::kAux; ++k)
            if (used[k]) {
                QK_CUDA_TRY(cudaEventRecord(c->join_ev[k], c->aux[k]));
                QK_CUDA_TRY(cudaStreamWaitEvent(s, c->join_ev[k], 0));
            }
    finalize_kernel<<<(n * n + 255) / 256, 256, 0, s>>>(A, n, o);
    QK_CUDA_TRY(cudaGetLastError());
    c->last_quart = nq;
    c->last_primq = npq;
    c->last_launches = c->launches;   // one launch per class (never the merged s/p kernel)
    return QK_OK;
}

}  // namespace qk


// ------------------------------------------------------------------ batches
// Many molecules in one Fock build.  Per call the host writes one staging block
// -- the molecules' DevData, their BatchMol records and every class's segment
// table -- into pinned memory (two blocks, used in turn, each guarded by the
// event of its last copy), copies it to the device with one cudaMemcpyAsync, and
// enqueues on the caller's stream: counters memset, batch_prep_kernel, the class
// kernels (FP64 and FP32 parts, one after another), batch_finalize_kernel.
struct qk_batch {
    int device = 0;
    std::mutex mu;
    int num_sms = 148;
    int bps[2 * qk::kNumClasses] = {};        // resident blocks per SM: FP64 kernels, then FP32 ones
    static constexpr int kStage = 2;
    char* h_stage[kStage] = {};
    size_t h_cap[kStage] = {};
    cudaEvent_t stage_ev[kStage] = {};
    int stage_next = 0;
    qk::DevBuf<char> d_stage;
    qk::DevBuf<int> d_counters;
    cudaEvent_t done_ev = nullptr;            // end of the previous build (orders reuse of d_stage)
    bool done_recorded = false;
    int reserve_sms = 0;                      // SMs the class kernels leave to other work
};

using namespace qk;

// =========================================================================== C ABI
extern "C" {

const char* qk_status_string(int s) {
    switch (s) {
        case QK_OK: return "ok";
        case QK_ERR_NO_DEVICE: return "no CUDA device";
        case QK_ERR_INVALID_ARG: return "invalid argument";
        case QK_ERR_NOT_READY: return "required upload missing";
        case QK_ERR_CUDA: return "CUDA error";
        case QK_ERR_OUT_OF_MEMORY: return "device out of memory";
        case QK_ERR_UNSUPPORTED: return "unsupported input";
        case QK_ERR_BASIS_LAYOUT: return "basis arrays do not follow QUICK's layout";
        default: return "unknown status";
    }
}

int qk_last_status(void) { return g_last_status.load(); }

int qk_set_maxprim(int maxprim) {
    if (maxprim < 1 || maxprim > kMaxPrimShell) return fail(QK_ERR_INVALID_ARG, "maxprim out of range");
    g_maxprim_default = maxprim;
    if (g_default) g_default->maxprim = maxprim;
    return QK_OK;
}

int qk_max_l(void) { return kMaxL; }

qk_ctx* qk_create(int device, int* status) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        if (status) *status = fail(QK_ERR_NO_DEVICE, "no CUDA device");
        return nullptr;
    }
    if (device < 0 || device >= ndev) {
        if (status) *status = fail(QK_ERR_INVALID_ARG, "device index out of range");
        return nullptr;
    }
    if (cudaSetDevice(device) != cudaSuccess) {
        if (status) *status = fail(QK_ERR_CUDA, "cudaSetDevice failed");
        return nullptr;
    }
    qk_ctx* c = new qk_ctx();
    c->device = device;
    c->maxprim = g_maxprim_default;
    cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
    // the context's own stream (tables, work lists, Schwarz bounds) at the highest
    // priority: a set-up that runs beside other contexts' long Fock builds gets the
    // SMs as soon as one of their kernels ends
    int prio_lo = 0, prio_hi = 0;
    cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
    if (cudaStreamCreateWithPriority(&c->stream, cudaStreamNonBlocking, prio_hi) != cudaSuccess) {
        delete c;
        if (status) *status = fail(QK_ERR_CUDA, "stream creation failed");
        return nullptr;
    }
    // the tables are the same for every context: computed once per process
    static std::once_flag once;
    static std::vector<double> tab, rows;
    std::call_once(once, [] {
        tab = boys_table();
        rows = boys_row_tables(tab);
    });
    if (c->d_boys.upload(tab, c->stream) != cudaSuccess || c->d_boys8.upload(rows, c->stream) != cudaSuccess ||
        cudaStreamSynchronize(c->stream) != cudaSuccess) {
        cudaStreamDestroy(c->stream);
        delete c;
        if (status) *status = fail(QK_ERR_CUDA, "Boys table upload failed");
        return nullptr;
    }
    if (status) *status = QK_OK;
    return c;
}

int qk_destroy(qk_ctx* c) {
    if (!c) return QK_OK;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    for (auto& e : c->ev)
        if (e) cudaEventDestroy(e);
    for (auto& a : c->aux)
        if (a) cudaStreamDestroy(a);
    for (auto& e : c->join_ev)
        if (e) cudaEventDestroy(e);
    if (c->fork_ev) cudaEventDestroy(c->fork_ev);
    cudaStreamDestroy(c->stream);
    delete c;
    return QK_OK;
}

qk_ctx* qk_default_ctx(void) {
    std::lock_guard<std::mutex> g(g_default_mu);
    if (!g_default) {
        int st = 0;
        g_default = qk_create(g_default_device, &st);
    }
    return g_default;
}

int qk_set_basis(qk_ctx* c, int natom, const double* xyz, int nshell, int nbasis, int jbasis,
                 const int* kstart, const int* katom, const int* kprim, const int* Ksumtype,
                 const int* Qstart, const int* Qfinal, const int* Qsbasis, const int* Qfbasis,
                 const double* gccoeff, const double* cons, const double* gcexpo, const int* KLMN,
                 int maxprim) {
    if (!c || natom <= 0 || nshell <= 0 || nbasis <= 0 || jbasis <= 0 || !xyz || !kstart || !katom ||
        !kprim || !Ksumtype || !Qstart || !Qfinal || !Qsbasis || !gccoeff || !cons || !gcexpo || !KLMN)
        return fail(QK_ERR_INVALID_ARG, "qk_set_basis: missing argument");
    if (maxprim <= 0) maxprim = c->maxprim;
    std::lock_guard<std::mutex> g(c->mu);
    cudaSetDevice(c->device);
    c->natom = natom; c->nshell = nshell; c->nbasis = nbasis; c->jbasis = jbasis;
    c->xyz.assign(xyz, xyz + 3 * natom);
    c->qsh.clear();
    c->shell_f0.assign(nshell, 0);
    c->shell_f1.assign(nshell, 0);
    c->shell_prim0.assign(nshell, 0);
    for (int s = 0; s < nshell; ++s) {
        const int np = kprim[s];
        if (np <= 0 || np > maxprim || np > kMaxPrimShell) return fail(QK_ERR_UNSUPPORTED, "contraction too long");
        if (Qfinal[s] > kMaxL) return fail(QK_ERR_UNSUPPORTED, "shell angular momentum above the compiled maximum");
        const int fbase = Ksumtype[s] - 1;
        c->shell_f0[s] = fbase + Qsbasis[s + nshell * Qstart[s]];
        c->shell_f1[s] = fbase + Qfbasis[s + nshell * Qfinal[s]] + 1;
        c->shell_prim0[s] = kstart[s] - 1;
        for (int L = Qstart[s]; L <= Qfinal[s]; ++L) {
            Qsh q{};
            q.L = L; q.parent = s; q.atom = katom[s] - 1; q.nprim = np; q.prim0 = kstart[s] - 1;
            q.f0 = fbase + Qsbasis[s + nshell * L];
            if (q.atom < 0 || q.atom >= natom || q.f0 < 0 || q.f0 + ncart(L) > nbasis)
                return fail(QK_ERR_INVALID_ARG, "shell index out of range");
            // contraction coefficient of the angular part L: gccoeff(k, Ksumtype + L)
            // (the column get_eri_precomputables uses, src/modules/include/eri.fh:132-137)
            const int col = fbase + L;
            for (int k = 0; k < np; ++k) {
                q.coef[k] = gccoeff[k + (size_t)maxprim * col];
                q.expo[k] = gcexpo[k + (size_t)maxprim * col];
            }
            for (int k = 0; k < ncart(L); ++k) {
                int e[3];
                cart_of(L, k, e);
                const int f = q.f0 + k;
                if (KLMN[3 * f] != e[0] || KLMN[3 * f + 1] != e[1] || KLMN[3 * f + 2] != e[2])
                    return fail(QK_ERR_BASIS_LAYOUT, "KLMN order differs from QUICK's convention");
                if (std::fabs(cons[f] - cons_expected(e)) > 1e-12)
                    return fail(QK_ERR_BASIS_LAYOUT, "cons factors differ from QUICK's convention");
            }
            c->qsh.push_back(q);
        }
    }
    std::vector<int> q_atom, q_f0, q_parent, q_ltop, q_prim0, q_nprim;
    for (auto& q : c->qsh) {
        q_atom.push_back(q.atom); q_f0.push_back(q.f0); q_parent.push_back(q.parent);
        q_ltop.push_back(Qfinal[q.parent]);
        q_prim0.push_back(q.prim0); q_nprim.push_back(q.nprim);
    }
    cudaStream_t s = c->stream;
    QK_CUDA_TRY(c->d_xyz.upload(c->xyz, s));
    QK_CUDA_TRY(c->d_q_atom.upload(q_atom, s));
    QK_CUDA_TRY(c->d_q_f0.upload(q_f0, s));
    QK_CUDA_TRY(c->d_q_parent.upload(q_parent, s));
    QK_CUDA_TRY(c->d_q_ltop.upload(q_ltop, s));
    c->q_ltop_h = q_ltop;
    QK_CUDA_TRY(c->d_q_prim0.upload(q_prim0, s));
    QK_CUDA_TRY(c->d_q_nprim.upload(q_nprim, s));
    QK_CUDA_TRY(c->d_shell_f0.upload(c->shell_f0, s));
    QK_CUDA_TRY(c->d_shell_f1.upload(c->shell_f1, s));
    QK_CUDA_TRY(cudaStreamSynchronize(s));
    c->have_basis = true;
    c->have_schwarz = false;
    c->pairs_dirty = true;
    return QK_OK;
}

int qk_set_schwarz(qk_ctx* c, const double* Y, const double* cp) {
    if (!c || !Y || !cp) return fail(QK_ERR_INVALID_ARG, "qk_set_schwarz: missing argument");
    std::lock_guard<std::mutex> g(c->mu);
    if (!c->have_basis) return fail(QK_ERR_NOT_READY, "basis not uploaded");
    const int ns = c->nshell, jb = c->jbasis;
    c->Ycut.assign((size_t)ns * ns, 0.0);
    c->cutprim.assign((size_t)jb * jb, 0.0);
    // The reference fills cutPrim(i,j) for shell(i) <= shell(j) only
    // (src/modules/quick_cutoff_module.f90:205-215); reads are orientation-free here.
    for (int i = 0; i < ns; ++i)
        for (int j = 0; j < ns; ++j)
            c->Ycut[(size_t)i * ns + j] = std::max(Y[i + (size_t)ns * j], Y[j + (size_t)ns * i]);
    for (int i = 0; i < jb; ++i)
        for (int j = 0; j < jb; ++j)
            c->cutprim[(size_t)i * jb + j] = std::max(cp[i + (size_t)jb * j], cp[j + (size_t)jb * i]);
    c->have_schwarz = true;
    c->pairs_dirty = true;
    return QK_OK;
}

int qk_schwarz(qk_ctx* c, double* Yout, double* cpout) {
    if (!c) return fail(QK_ERR_INVALID_ARG, "null context");
    std::vector<double> Y, cp;
    {
        std::lock_guard<std::mutex> g(c->mu);
        if (!c->have_basis) return fail(QK_ERR_NOT_READY, "basis not uploaded");
        cudaSetDevice(c->device);
        build_pairs(c, false);
        int st = upload_pairs(c);
        if (st) return st;
        c->pairs_dirty = true;
        const int ns = c->nshell, jb = c->jbasis;
        // scratch kept in the context: freeing device memory synchronises the whole GPU
        DevBuf<unsigned long long>& dY = c->d_schwarz_Y;
        DevBuf<unsigned long long>& dcp = c->d_schwarz_cp;
        QK_CUDA_TRY(dY.reserve((size_t)ns * ns));
        QK_CUDA_TRY(dcp.reserve((size_t)jb * jb));
        QK_CUDA_TRY(cudaMemsetAsync(dY.p, 0, sizeof(unsigned long long) * ns * ns, c->stream));
        QK_CUDA_TRY(cudaMemsetAsync(dcp.p, 0, sizeof(unsigned long long) * jb * jb, c->stream));
        DevData d = make_devdata(c);
        const PairTable& T = c->pairs;
        // one work list per pair class
        int lmax = kMaxL;
        std::vector<std::vector<int2>> wl((lmax + 1) * (lmax + 1));
        for (int p = 0; p < (int)T.qa.size(); ++p) {
            const int La = c->qsh[T.qa[p]].L, Lb = c->qsh[T.qb[p]].L;
            auto& v = wl[La * (lmax + 1) + Lb];
            v.push_back(make_int2(p, -1));
            for (int k = 0; k < T.npp[p]; ++k) v.push_back(make_int2(p, k));
        }
        DevBuf<int2>* dwl = c->d_schwarz_work;
#define QK_SCHWARZ(a, b)                                                                          \
        {                                                                                         \
            auto& v = wl[a * (lmax + 1) + b];                                                     \
            if (!v.empty()) {                                                                     \
                auto& dv = dwl[a * (lmax + 1) + b];                                               \
                QK_CUDA_TRY(dv.upload(v, c->stream));                                             \
                QK_CUDA_TRY((launch_schwarz<a, b>(d, dv.p, (int)v.size(), c->d_q_prim0.p,          \
                                                  c->d_q_nprim.p, ns, jb, dY.p, dcp.p, c->num_sms, \
                                                  c->stream)));                                    \
            }                                                                                     \
        }
        QK_PAIR_CLASS_LIST(QK_SCHWARZ)
#undef QK_SCHWARZ
        std::vector<unsigned long long> hY((size_t)ns * ns), hcp((size_t)jb * jb);
        QK_CUDA_TRY(cudaMemcpyAsync(hY.data(), dY.p, hY.size() * 8, cudaMemcpyDeviceToHost, c->stream));
        QK_CUDA_TRY(cudaMemcpyAsync(hcp.data(), dcp.p, hcp.size() * 8, cudaMemcpyDeviceToHost, c->stream));
        QK_CUDA_TRY(cudaStreamSynchronize(c->stream));
        Y.resize(hY.size());
        cp.resize(hcp.size());
        for (size_t i = 0; i < hY.size(); ++i) {
            double v;
            std::memcpy(&v, &hY[i], 8);
            Y[i] = std::sqrt(v);
        }
        for (size_t i = 0; i < hcp.size(); ++i) {
            double v;
            std::memcpy(&v, &hcp[i], 8);
            cp[i] = std::sqrt(v);
        }
    }
    // Y and cutprim are symmetric, so row- and column-major agree
    if (Yout) std::memcpy(Yout, Y.data(), Y.size() * 8);
    if (cpout) std::memcpy(cpout, cp.data(), cp.size() * 8);
    return qk_set_schwarz(c, Y.data(), cp.data());
}

int qk_set_cutoffs(qk_ctx* c, double integralCutoff, double primLimit) {
    if (!c || !(integralCutoff > 0.0) || !(primLimit > 0.0)) return fail(QK_ERR_INVALID_ARG, "bad cutoffs");
    std::lock_guard<std::mutex> g(c->mu);
    c->integralCutoff = integralCutoff;
    c->primLimit = primLimit;
    return QK_OK;
}

int qk_set_precision(qk_ctx* c, double fp32_bound) {
    if (!c || !(fp32_bound >= 0.0)) return fail(QK_ERR_INVALID_ARG, "bad precision bound");
    std::lock_guard<std::mutex> g(c->mu);
    c->fp32_bound = fp32_bound;
    return QK_OK;
}

int qk_set_boys(qk_ctx* c, int mode) {
    if (!c || mode < 0 || mode > 2) return fail(QK_ERR_INVALID_ARG, "qk_set_boys: mode must be 0, 1 or 2");
    std::lock_guard<std::mutex> g(c->mu);
    c->boys_mode = mode;
    return QK_OK;
}

int qk_last_work_mixed(qk_ctx* c, long long* quartets_fp32) {
    if (!c || !quartets_fp32) return fail(QK_ERR_INVALID_ARG, "null argument");
    long long q = 0;
    for (int ci = 0; ci < kNumClasses; ++ci) q += c->work[ci].nquart32;
    *quartets_fp32 = q;
    return QK_OK;
}

int qk_density_cutoff_device(qk_ctx* c, const double* D, double* cutmat, void* stream) {
    if (!c || !D || !cutmat) return fail(QK_ERR_INVALID_ARG, "null argument");
    std::lock_guard<std::mutex> g(c->mu);
    if (!c->have_basis) return fail(QK_ERR_NOT_READY, "basis not uploaded");
    cudaSetDevice(c->device);
    cudaStream_t s = (cudaStream_t)stream;   // NULL = the CUDA default stream
    const int ns = c->nshell;
    density_cutoff_kernel<<<(ns * ns + 127) / 128, 128, 0, s>>>(D, c->nbasis, ns, c->d_shell_f0.p,
                                                                 c->d_shell_f1.p, cutmat);
    QK_CUDA_TRY(cudaGetLastError());
    return QK_OK;
}

int qk_fock2e_device(qk_ctx* c, const double* D, const double* cutmat, double* o, void* stream) {
    if (!c || !D || !o) return fail(QK_ERR_INVALID_ARG, "null argument");
    std::lock_guard<std::mutex> g(c->mu);
    cudaSetDevice(c->device);
    // NULL = the CUDA default stream, as everywhere in CUDA
    return fock2e_device(c, D, cutmat, o, (cudaStream_t)stream);
}

int qk_fock2e_host(qk_ctx* c, const double* D, const double* cutmat, double* o) {
    if (!c || !D || !o) return fail(QK_ERR_INVALID_ARG, "null argument");
    std::lock_guard<std::mutex> g(c->mu);
    cudaSetDevice(c->device);
    const int n = c->nbasis, ns = c->nshell;
    cudaStream_t s = c->stream;
    QK_CUDA_TRY(c->d_D.reserve((size_t)n * n));
    QK_CUDA_TRY(c->d_o.reserve((size_t)n * n));
    // o goes up with D and comes back with G added on the device: no host-side
    // staging buffer and no host loop
    QK_CUDA_TRY(cudaMemcpyAsync(c->d_D.p, D, sizeof(double) * n * n, cudaMemcpyHostToDevice, s));
    QK_CUDA_TRY(cudaMemcpyAsync(c->d_o.p, o, sizeof(double) * n * n, cudaMemcpyHostToDevice, s));
    const double* cm = nullptr;
    if (cutmat) {
        QK_CUDA_TRY(c->d_cutmat.reserve((size_t)ns * ns));
        QK_CUDA_TRY(cudaMemcpyAsync(c->d_cutmat.p, cutmat, sizeof(double) * ns * ns, cudaMemcpyHostToDevice, s));
        cm = c->d_cutmat.p;
    }
    int st = fock2e_device(c, c->d_D.p, cm, c->d_o.p, s);
    if (st) return st;
    QK_CUDA_TRY(cudaMemcpyAsync(o, c->d_o.p, sizeof(double) * n * n, cudaMemcpyDeviceToHost, s));
    QK_CUDA_TRY(cudaStreamSynchronize(s));
    return QK_OK;
}

int qk_fock2e_uhf_device(qk_ctx* c, const double* Da, const double* Db, const double* cutmat, double* oa, double* ob,
                         void* stream) {
    if (!c || !Da || !Db || !oa || !ob) return fail(QK_ERR_INVALID_ARG, "null argument");
    std::lock_guard<std::mutex> g(c->mu);
    if (cudaSetDevice(c->device) != cudaSuccess) return fail(QK_ERR_CUDA, "cudaSetDevice");
    return fock2e_uhf_device(c, Da, Db, cutmat, oa, ob, (cudaStream_t)stream);
}

int qk_fock2e_uhf_host(qk_ctx* c, const double* Da, const double* Db, const double* cutmat, double* oa, double* ob) {
    if (!c || !Da || !Db || !oa || !ob) return fail(QK_ERR_INVALID_ARG, "null argument");
    std::lock_guard<std::mutex> g(c->mu);
    if (cudaSetDevice(c->device) != cudaSuccess) return fail(QK_ERR_CUDA, "cudaSetDevice");
    const int n = c->nbasis, ns = c->nshell;
    const size_t nn = (size_t)n * n;
    cudaStream_t s = c->stream;
    // device copies: Da in d_D, oa in d_o, Db and ob in the second half of d_D / d_o
    QK_CUDA_TRY(c->d_D.reserve(2 * nn));
    QK_CUDA_TRY(c->d_o.reserve(2 * nn));
    QK_CUDA_TRY(cudaMemcpyAsync(c->d_D.p, Da, sizeof(double) * nn, cudaMemcpyHostToDevice, s));
    QK_CUDA_TRY(cudaMemcpyAsync(c->d_D.p + nn, Db, sizeof(double) * nn, cudaMemcpyHostToDevice, s));
    QK_CUDA_TRY(cudaMemcpyAsync(c->d_o.p, oa, sizeof(double) * nn, cudaMemcpyHostToDevice, s));
    QK_CUDA_TRY(cudaMemcpyAsync(c->d_o.p + nn, ob, sizeof(double) * nn, cudaMemcpyHostToDevice, s));
    const double* cm = nullptr;
    if (cutmat) {
        QK_CUDA_TRY(c->d_cutmat.reserve((size_t)ns * ns));
        QK_CUDA_TRY(cudaMemcpyAsync(c->d_cutmat.p, cutmat, sizeof(double) * ns * ns, cudaMemcpyHostToDevice, s));
        cm = c->d_cutmat.p;
    }
    int st = fock2e_uhf_device(c, c->d_D.p, c->d_D.p + nn, cm, c->d_o.p, c->d_o.p + nn, s);
    if (st) return st;
    QK_CUDA_TRY(cudaMemcpyAsync(oa, c->d_o.p, sizeof(double) * nn, cudaMemcpyDeviceToHost, s));
    QK_CUDA_TRY(cudaMemcpyAsync(ob, c->d_o.p + nn, sizeof(double) * nn, cudaMemcpyDeviceToHost, s));
    QK_CUDA_TRY(cudaStreamSynchronize(s));
    return QK_OK;
}

// Allocation-free variant of qk_fock2e_device for callers that may not allocate
// device memory when they run a Fock build; see the comment at g_noalloc_scratch.
// Its first call on a device looks up the scratch array's device address (one
// cudaGetSymbolAddress); make that first call before any stream capture.  All
// calls share the one scratch array, so calls that overlap on the GPU race:
// serialise them (one stream, or events between streams).
int qk_fock2e_device_noalloc(qk_ctx* c, const double* D, const double* cutmat, double* o, void* stream) {
    if (!c || !D || !o) return fail(QK_ERR_INVALID_ARG, "null argument");
    std::lock_guard<std::mutex> g(c->mu);
    if (cudaSetDevice(c->device) != cudaSuccess) return fail(QK_ERR_CUDA, "cudaSetDevice");
    return fock2e_device_noalloc(c, D, cutmat, o, (cudaStream_t)stream);
}


// ------------------------------------------------------------- sharded builds (C ABI)
int qk_set_shard(qk_ctx* c, int rank, int count) {
    if (!c || count < 1 || rank < 0 || rank >= count) return fail(QK_ERR_INVALID_ARG, "qk_set_shard: bad rank/count");
    std::lock_guard<std::mutex> g(c->mu);
    if (c->shard_rank != rank || c->shard_count != count) {
        c->shard_rank = rank;
        c->shard_count = count;
        c->pairs_dirty = true;
    }
    return QK_OK;
}

int qk_fock2e_device_accumulate(qk_ctx* c, const double* D, const double* cutmat, long long* A, void* stream) {
    if (!c || !D || !A) return fail(QK_ERR_INVALID_ARG, "null argument");
    std::lock_guard<std::mutex> g(c->mu);
    if (cudaSetDevice(c->device) != cudaSuccess) return fail(QK_ERR_CUDA, "cudaSetDevice");
    return fock2e_device(c, D, cutmat, nullptr, (cudaStream_t)stream, reinterpret_cast<unsigned long long*>(A));
}

int qk_finalize_fixed(const long long* A, int n, double* o, void* stream) {
    if (!A || !o || n < 1) return fail(QK_ERR_INVALID_ARG, "qk_finalize_fixed: bad argument");
    finalize_kernel<<<(n * n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
        reinterpret_cast<const unsigned long long*>(A), n, o);
    QK_CUDA_TRY(cudaGetLastError());
    return QK_OK;
}


// ------------------------------------------------------------- batches (C ABI)
qk_batch* qk_batch_create(int device, int* status) {
    if (cudaSetDevice(device) != cudaSuccess) {
        if (status) *status = fail(QK_ERR_NO_DEVICE, "qk_batch_create: cudaSetDevice");
        return nullptr;
    }
    qk_batch* b = new qk_batch();
    b->device = device;
    cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, device);
    bool ok = cudaEventCreateWithFlags(&b->done_ev, cudaEventDisableTiming) == cudaSuccess;
    for (int k = 0; ok && k < qk_batch::kStage; ++k)
        ok = cudaEventCreateWithFlags(&b->stage_ev[k], cudaEventDisableTiming) == cudaSuccess;
    for (int slot = 0; ok && slot < 2 * kNumClasses; ++slot) {
        const ClassEntry& ce = g_classes[slot % kNumClasses];
        const bool fp32 = slot >= kNumClasses;
        const int wpb = ce.coop ? ce.coop_warps : kWarpsPerBlock;
        if (ce.smem > 48 * 1024)
            ok = cudaFuncSetAttribute(ce.kernel_batch(fp32), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)ce.smem) == cudaSuccess;
        ok = ok && cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b->bps[slot], ce.kernel_batch(fp32), 32 * wpb,
                                                                 ce.smem) == cudaSuccess && b->bps[slot] >= 1;
    }
    if (!ok || b->d_counters.reserve(2 * kNumClasses) != cudaSuccess) {
        qk_batch_destroy(b);
        if (status) *status = fail(QK_ERR_CUDA, "qk_batch_create");
        return nullptr;
    }
    if (status) *status = QK_OK;
    return b;
}

int qk_batch_destroy(qk_batch* b) {
    if (!b) return QK_OK;
    cudaSetDevice(b->device);
    cudaDeviceSynchronize();
    for (int k = 0; k < qk_batch::kStage; ++k) {
        if (b->stage_ev[k]) cudaEventDestroy(b->stage_ev[k]);
        if (b->h_stage[k]) cudaFreeHost(b->h_stage[k]);
    }
    if (b->done_ev) cudaEventDestroy(b->done_ev);
    delete b;
    return QK_OK;
}

namespace {
size_t align16(size_t x) { return (x + 15) & ~size_t(15); }
}

int qk_batch_reserve_sms(qk_batch* b, int sms) {
    if (!b || sms < 0) return fail(QK_ERR_INVALID_ARG, "qk_batch_reserve_sms");
    std::lock_guard<std::mutex> g(b->mu);
    b->reserve_sms = std::min(sms, b->num_sms - 1);
    return QK_OK;
}

int qk_batch_fock2e(qk_batch* b, int n, qk_ctx* const* ctxs, const double* const* D, const double* const* cutmat,
                    double* const* o, void* stream) {
    if (!b || n <= 0 || !ctxs || !D || !o) return fail(QK_ERR_INVALID_ARG, "qk_batch_fock2e: null argument");
    if (n > 65535) return fail(QK_ERR_INVALID_ARG, "qk_batch_fock2e: more than 65535 molecules");
    std::lock_guard<std::mutex> g(b->mu);
    if (cudaSetDevice(b->device) != cudaSuccess) return fail(QK_ERR_CUDA, "cudaSetDevice");
    cudaStream_t s = (cudaStream_t)stream;
    // per molecule: tables ready, accumulator and screen buffers sized
    long long max_nn = 0;
    for (int m = 0; m < n; ++m) {
        qk_ctx* c = ctxs[m];
        if (!c || !D[m] || !o[m]) return fail(QK_ERR_INVALID_ARG, "qk_batch_fock2e: null molecule entry");
        if (c->device != b->device) return fail(QK_ERR_INVALID_ARG, "qk_batch_fock2e: context on another device");
        if (c->shard_count > 1) return fail(QK_ERR_INVALID_ARG, "qk_batch_fock2e: context is sharded (qk_set_shard)");
        for (int j = 0; j < m; ++j)
            if (ctxs[j] == c)
                return fail(QK_ERR_INVALID_ARG, "qk_batch_fock2e: a context appears twice (its accumulator is shared)");
        std::lock_guard<std::mutex> gc(c->mu);
        int st = ensure_pairs(c);
        if (st) return st;
        QK_CUDA_TRY(c->d_A.reserve((size_t)c->nbasis * c->nbasis));
        if (!(cutmat && cutmat[m])) QK_CUDA_TRY(c->d_cutmat.reserve((size_t)c->nshell * c->nshell));
        max_nn = std::max<long long>(max_nn, (long long)c->nbasis * c->nbasis);
    }
    // staging block: [DevData x n][BatchMol x n][BatchSeg per slot]; slot ci = the
    // FP64 items of class ci, slot kNumClasses + ci = its FP32 items (mixed form)
    constexpr int kSlots = 2 * kNumClasses;
    auto part_range = [&](const ClassWork& W, int slot, int* first, int* count) {
        *first = slot < kNumClasses ? 0 : W.n64;
        *count = slot < kNumClasses ? W.n64 : W.n_items - W.n64;
    };
    int seg_count[kSlots], seg_off[kSlots], total_items[kSlots];
    int nseg_all = 0;
    for (int slot = 0; slot < kSlots; ++slot) {
        seg_off[slot] = nseg_all;
        seg_count[slot] = 0;
        long long tot = 0;
        for (int m = 0; m < n; ++m) {
            int f, cnt;
            part_range(ctxs[m]->work[slot % kNumClasses], slot, &f, &cnt);
            if (cnt > 0) {
                ++seg_count[slot];
                tot += cnt;
            }
        }
        if (tot > INT_MAX) return fail(QK_ERR_INVALID_ARG, "qk_batch_fock2e: too many work items in one class");
        total_items[slot] = (int)tot;
        nseg_all += seg_count[slot];
    }
    const size_t off_mol = align16(sizeof(DevData) * n);
    const size_t off_seg = off_mol + align16(sizeof(BatchMol) * n);
    const size_t bytes = off_seg + sizeof(BatchSeg) * (size_t)std::max(nseg_all, 1);
    const int k = b->stage_next;
    b->stage_next = (k + 1) % qk_batch::kStage;
    QK_CUDA_TRY(cudaEventSynchronize(b->stage_ev[k]));   // its previous copy has been read
    if (b->h_cap[k] < bytes) {
        if (b->h_stage[k]) cudaFreeHost(b->h_stage[k]);
        b->h_stage[k] = nullptr;
        b->h_cap[k] = 0;
        QK_CUDA_TRY(cudaHostAlloc((void**)&b->h_stage[k], bytes * 2, cudaHostAllocDefault));
        b->h_cap[k] = bytes * 2;
    }
    char* hs = b->h_stage[k];
    DevData* hd = (DevData*)hs;
    BatchMol* hm = (BatchMol*)(hs + off_mol);
    BatchSeg* hg = (BatchSeg*)(hs + off_seg);
    for (int m = 0; m < n; ++m) {
        qk_ctx* c = ctxs[m];
        const bool own_cut = !(cutmat && cutmat[m]);
        DevData d = make_devdata(c);
        d.D = D[m];
        d.cutmat = own_cut ? c->d_cutmat.p : cutmat[m];
        d.A = c->d_A.p;
        d.stats = nullptr;
        hd[m] = d;
        hm[m] = BatchMol{D[m], own_cut ? c->d_cutmat.p : nullptr, c->d_A.p, o[m], c->d_shell_f0.p,
                         c->d_shell_f1.p, c->nbasis, c->nshell};
    }
    // device addresses of the staged arrays (d_stage may grow: wait for the last build first)
    if (b->done_recorded) QK_CUDA_TRY(cudaStreamWaitEvent(s, b->done_ev, 0));
    if (b->d_stage.cap < bytes) {
        if (b->done_recorded) QK_CUDA_TRY(cudaEventSynchronize(b->done_ev));
        QK_CUDA_TRY(b->d_stage.reserve(bytes * 2));
    }
    char* ds = b->d_stage.p;
    const DevData* dd = (const DevData*)ds;
    const BatchMol* dm = (const BatchMol*)(ds + off_mol);
    const BatchSeg* dg = (const BatchSeg*)(ds + off_seg);
    for (int slot = 0; slot < kSlots; ++slot) {
        BatchSeg* sg = hg + seg_off[slot];
        int at = 0, ns = 0;
        for (int m = 0; m < n; ++m) {
            const ClassWork& W = ctxs[m]->work[slot % kNumClasses];
            int f, cnt;
            part_range(W, slot, &f, &cnt);
            if (cnt <= 0) continue;
            sg[ns++] = BatchSeg{W.d_items + f, at, m};
            at += cnt;
        }
    }
    QK_CUDA_TRY(cudaMemcpyAsync(ds, hs, bytes, cudaMemcpyHostToDevice, s));
    QK_CUDA_TRY(cudaEventRecord(b->stage_ev[k], s));
    QK_CUDA_TRY(cudaMemsetAsync(b->d_counters.p, 0, sizeof(int) * kSlots, s));
    const int chunks = (int)std::min<long long>(64, std::max<long long>(1, (max_nn + 2047) / 2048));
    batch_prep_kernel<<<dim3(chunks, n), 256, 0, s>>>(dm);
    QK_CUDA_TRY(cudaGetLastError());
    // class launches one after another on the caller's stream (faster than
    // concurrent launches that each fill the GPU), cooperative classes first
    int order[kSlots], no = 0;
    for (int slot = 0; slot < kSlots; ++slot)
        if (total_items[slot] > 0) order[no++] = slot;
    std::stable_sort(order, order + no, [&](int x, int y) {
        const ClassEntry& cx = g_classes[x % kNumClasses];
        const ClassEntry& cy = g_classes[y % kNumClasses];
        if (cx.coop != cy.coop) return cx.coop;
        return (double)total_items[x] * cx.prim_flops > (double)total_items[y] * cy.prim_flops;
    });
    for (int i = 0; i < no; ++i) {
        const int slot = order[i];
        const ClassEntry& ce = g_classes[slot % kNumClasses];
        const int wpb = ce.coop ? ce.coop_warps : kWarpsPerBlock;
        const long long need = ((long long)total_items[slot] + wpb - 1) / wpb;
        const int sms = std::max(1, b->num_sms - b->reserve_sms);
        const int grid = (int)std::min<long long>((long long)b->bps[slot] * sms, need);
        ce.fn_batch(slot >= kNumClasses, dim3(grid), dim3(32 * wpb), ce.smem, s, dd, dg + seg_off[slot],
                    seg_count[slot], total_items[slot], b->d_counters.p + slot);
        QK_CUDA_TRY(cudaGetLastError());
    }
    batch_finalize_kernel<<<dim3(chunks, n), 256, 0, s>>>(dm);
    QK_CUDA_TRY(cudaGetLastError());
    QK_CUDA_TRY(cudaEventRecord(b->done_ev, s));
    b->done_recorded = true;
    return QK_OK;
}

int qk_prepare(qk_ctx* c) {
    if (!c) return fail(QK_ERR_INVALID_ARG, "qk_prepare: null context");
    std::lock_guard<std::mutex> g(c->mu);
    if (cudaSetDevice(c->device) != cudaSuccess) return fail(QK_ERR_CUDA, "cudaSetDevice");
    return ensure_pairs(c);
}

int qk_device_bytes(qk_ctx* c, unsigned long long* total, unsigned long long* items) {
    if (!c) return fail(QK_ERR_INVALID_ARG, "qk_device_bytes: null context");
    std::lock_guard<std::mutex> g(c->mu);
    const PairTable& T = c->pairs;
    unsigned long long it = 0;
    it += c->d_items.bytes() + c->d_wl.bytes();
    unsigned long long t = it;
    for (size_t b : {T.d_qa.bytes(), T.d_qb.bytes(), T.d_pp0.bytes(), T.d_npp.bytes(), T.d_pps.bytes(),
                     T.d_Y.bytes(), T.d_zo.bytes(), T.d_kc.bytes(), T.d_pxy.bytes(), T.d_pzax.bytes(),
                     T.d_payz.bytes(), T.d_sh.bytes(), T.d_lt.bytes(), T.d_geo.bytes(), c->d_xyz.bytes(), c->d_boys.bytes(), c->d_boys8.bytes(), c->d_schwarz_Y.bytes(), c->d_schwarz_cp.bytes(), c->d_D.bytes(), c->d_cutmat.bytes(),
                     c->d_o.bytes(), c->d_q_atom.bytes(), c->d_q_f0.bytes(), c->d_q_parent.bytes(), c->d_q_ltop.bytes(),
                     c->d_q_prim0.bytes(), c->d_q_nprim.bytes(), c->d_shell_f0.bytes(), c->d_shell_f1.bytes(),
                     c->d_A.bytes(), c->d_A2.bytes(), c->d_uhf.bytes(), c->d_counters.bytes(), c->d_stats.bytes()})
        t += b;
    if (total) *total = t;
    if (items) *items = it;
    return QK_OK;
}

// kernel launches of one build with the current lists and settings
static int build_launches(const qk_ctx* c) {
    return (c->merge_sp && c->m_ready && !c->profile_events && !c->profile_stats) ? c->m_launches : c->launches;
}

int qk_last_work(qk_ctx* c, long long* quartets, long long* primq, int* launches) {
    if (!c) return fail(QK_ERR_INVALID_ARG, "null context");
    if (quartets) *quartets = c->last_quart;
    if (primq) *primq = c->last_primq;
    if (launches) *launches = c->last_launches ? c->last_launches : build_launches(c);
    return QK_OK;
}

int qk_launches_per_build(qk_ctx* c) { return c ? build_launches(c) : 0; }

int qk_set_merge_sp(qk_ctx* c, int on) {
    if (!c || (on != 0 && on != 1)) return fail(QK_ERR_INVALID_ARG, "qk_set_merge_sp: 0 or 1");
    std::lock_guard<std::mutex> g(c->mu);
    c->merge_sp = on == 1;
    c->m_ready = false;
    return QK_OK;
}

int qk_set_class_launch(qk_ctx* c, int ci, int warps_per_block, int blocks_per_sm) {
    if (!c || ci < 0 || ci >= kNumClasses) return fail(QK_ERR_INVALID_ARG, "qk_set_class_launch: class index");
    const ClassEntry& ce = g_classes[ci];
    const int maxw = ce.coop ? ce.coop_warps : kMaxLaneWarps;
    if (warps_per_block < 0 || warps_per_block > maxw || blocks_per_sm < 0 || blocks_per_sm > 64)
        return fail(QK_ERR_INVALID_ARG, "qk_set_class_launch: warps per block or blocks per SM out of range");
    std::lock_guard<std::mutex> g(c->mu);
    if (cudaSetDevice(c->device) != cudaSuccess) return fail(QK_ERR_CUDA, "cudaSetDevice");
    c->cls_wpb[ci] = warps_per_block;
    c->cls_bpsm[ci] = blocks_per_sm;
    if (c->work[ci].n_items > 0) return class_launch_shape(c, ci);
    return QK_OK;
}

int qk_class_launch(qk_ctx* c, int ci, int* warps_per_block, int* max_warps, int* blocks_per_sm, int* grid) {
    if (!c || ci < 0 || ci >= kNumClasses) return fail(QK_ERR_INVALID_ARG, "qk_class_launch: class index");
    const ClassEntry& ce = g_classes[ci];
    std::lock_guard<std::mutex> g(c->mu);
    const ClassWork& W = c->work[ci];
    if (warps_per_block)
        *warps_per_block = W.block > 0 ? W.block / 32
                                       : (c->cls_wpb[ci] > 0 ? c->cls_wpb[ci] : (ce.coop ? ce.coop_warps : kWarpsPerBlock));
    if (max_warps) *max_warps = ce.coop ? ce.coop_warps : kMaxLaneWarps;
    if (blocks_per_sm) *blocks_per_sm = c->cls_bpsm[ci];
    if (grid) *grid = W.n_items == 0 ? 0 : W.grid;
    return QK_OK;
}

int qk_stream_create(int device, int high_priority, void** stream) {
    if (!stream) return fail(QK_ERR_INVALID_ARG, "qk_stream_create: stream is NULL");
    *stream = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
        return fail(QK_ERR_INVALID_ARG, "qk_stream_create: device index out of range");
    int prev = 0;
    cudaGetDevice(&prev);
    if (cudaSetDevice(device) != cudaSuccess) return fail(QK_ERR_CUDA, "cudaSetDevice failed");
    int lo = 0, hi = 0;
    cudaDeviceGetStreamPriorityRange(&lo, &hi);
    cudaStream_t s = nullptr;
    cudaError_t e = cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, high_priority ? hi : lo);
    cudaSetDevice(prev);
    if (e != cudaSuccess) return fail(QK_ERR_CUDA, "qk_stream_create: stream creation failed");
    *stream = s;
    return QK_OK;
}

int qk_stream_destroy(void* stream) {
    if (!stream) return QK_OK;
    return cudaStreamDestroy(static_cast<cudaStream_t>(stream)) == cudaSuccess
               ? QK_OK : fail(QK_ERR_CUDA, "qk_stream_destroy failed");
}

int qk_set_worklist_builder(qk_ctx* c, int on_device) {
    if (!c || (on_device != 0 && on_device != 1)) return fail(QK_ERR_INVALID_ARG, "qk_set_worklist_builder: 0 or 1");
    std::lock_guard<std::mutex> g(c->mu);
    if (c->worklist_on_device != (on_device == 1)) {
        c->worklist_on_device = on_device == 1;
        c->pairs_dirty = true;
    }
    return QK_OK;
}

int qk_set_streams(qk_ctx* c, int nstreams) {
    if (!c || nstreams < 0 || nstreams > qk_ctx::kAux) return fail(QK_ERR_INVALID_ARG, "qk_set_streams: 0..4");
    std::lock_guard<std::mutex> g(c->mu);
    c->nstreams = nstreams;
    return QK_OK;
}

int qk_set_profiling(qk_ctx* c, int events, int stats) {
    if (!c) return fail(QK_ERR_INVALID_ARG, "null context");
    std::lock_guard<std::mutex> g(c->mu);
    cudaSetDevice(c->device);
    if (events && !c->ev[0])
        for (auto& e : c->ev) QK_CUDA_TRY(cudaEventCreate(&e));
    c->profile_events = events != 0;
    c->profile_stats = stats != 0;
    return QK_OK;
}

int qk_class_profile(qk_ctx* c, int max_classes, int* cls, float* ms, long long* q_listed,
                     long long* pq_listed, long long* q_done, long long* pq_done, double* prim_flops,
                     double* quartet_flops) {
    if (!c) return -fail(QK_ERR_INVALID_ARG, "null context");
    std::lock_guard<std::mutex> g(c->mu);
    cudaSetDevice(c->device);
    std::vector<unsigned long long> st(2 * kNumClasses, 0);
    if (c->profile_stats && c->d_stats.p) {
        if (cudaDeviceSynchronize() != cudaSuccess ||
            cudaMemcpy(st.data(), c->d_stats.p, st.size() * 8, cudaMemcpyDeviceToHost) != cudaSuccess)
            return -fail(QK_ERR_CUDA, "stats download");
    }
    const int n = std::min(max_classes, kNumClasses);
    for (int i = 0; i < n; ++i) {
        const ClassEntry& ce = g_classes[i];
        if (cls) { cls[4 * i] = ce.La; cls[4 * i + 1] = ce.Lb; cls[4 * i + 2] = ce.Lc; cls[4 * i + 3] = ce.Ld; }
        float t = 0.0f;
        if (c->profile_events && c->ev_recorded[i]) {
            if (cudaEventSynchronize(c->ev[2 * i + 1]) != cudaSuccess ||
                cudaEventElapsedTime(&t, c->ev[2 * i], c->ev[2 * i + 1]) != cudaSuccess)
                return -fail(QK_ERR_CUDA, "event timing");
        }
        if (ms) ms[i] = t;
        if (q_listed) q_listed[i] = c->work[i].nquart;
        if (pq_listed) pq_listed[i] = c->work[i].nprimq;
        if (q_done) q_done[i] = (long long)st[2 * i];
        if (pq_done) pq_done[i] = (long long)st[2 * i + 1];
        if (prim_flops) prim_flops[i] = ce.prim_flops;
        if (quartet_flops) quartet_flops[i] = ce.quartet_flops;
    }
    return n;
}

int qk_fp64_peak(int device, double* gflops) {
    if (!gflops) return fail(QK_ERR_INVALID_ARG, "null output");
    if (cudaSetDevice(device) != cudaSuccess) return fail(QK_ERR_CUDA, "cudaSetDevice");
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    DevBuf<double> out;
    QK_CUDA_TRY(out.reserve(1));
    cudaEvent_t e0, e1;
    QK_CUDA_TRY(cudaEventCreate(&e0));
    QK_CUDA_TRY(cudaEventCreate(&e1));
    const int blocks = sms * 8, threads = 256, iters = 2000;
    fp64_probe_kernel<<<blocks, threads>>>(out.p, 200, 0.999999, 1e-7);   // warm-up
    QK_CUDA_TRY(cudaGetLastError());
    float best = 1e30f;
    for (int r = 0; r < 5; ++r) {
        QK_CUDA_TRY(cudaEventRecord(e0));
        fp64_probe_kernel<<<blocks, threads>>>(out.p, iters, 0.999999, 1e-7);
        QK_CUDA_TRY(cudaEventRecord(e1));
        QK_CUDA_TRY(cudaEventSynchronize(e1));
        float t = 0.0f;
        QK_CUDA_TRY(cudaEventElapsedTime(&t, e0, e1));
        best = std::min(best, t);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    const double flops = 2.0 * 8 * 16 * (double)iters * blocks * threads;
    *gflops = flops / (best * 1e-3) * 1e-9;
    return QK_OK;
}


int qk_boys(qk_ctx* c, int M, const double* T, int n, double* F_rows, double* F_one) {
    if (!c || !T || !F_rows || !F_one || n < 1 || M < 0 || M > 4 * kMaxL)
        return fail(QK_ERR_INVALID_ARG, "qk_boys: bad argument");
    for (int i = 0; i < n; ++i)
        if (!(T[i] >= 0.0)) return fail(QK_ERR_INVALID_ARG, "qk_boys: T must be >= 0");
    std::lock_guard<std::mutex> g(c->mu);
    if (cudaSetDevice(c->device) != cudaSuccess) return fail(QK_ERR_CUDA, "cudaSetDevice");
    cudaStream_t s = c->stream;
    const size_t nout = (size_t)n * (M + 1);
    DevBuf<double> dT, dr, d1;
    QK_CUDA_TRY(dT.reserve(n));
    QK_CUDA_TRY(dr.reserve(nout));
    QK_CUDA_TRY(d1.reserve(nout));
    QK_CUDA_TRY(cudaMemcpyAsync(dT.p, T, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    const double2* rows8 = (const double2*)c->d_boys8.p;
    const double* tab = c->d_boys.p;
    cudaError_t e = cudaErrorInvalidValue;
    switch (M) {
#define QK_BOYS_CASE(m) case m: e = launch_boys_probe<m>(dT.p, n, rows8, tab, c->boys_mode, dr.p, d1.p, s); break;
        QK_BOYS_CASE(0) QK_BOYS_CASE(1) QK_BOYS_CASE(2) QK_BOYS_CASE(3) QK_BOYS_CASE(4)
#if QK_MAX_L >= 2
        QK_BOYS_CASE(5) QK_BOYS_CASE(6) QK_BOYS_CASE(7) QK_BOYS_CASE(8)
#endif
#if QK_MAX_L >= 3
        QK_BOYS_CASE(9) QK_BOYS_CASE(10) QK_BOYS_CASE(11) QK_BOYS_CASE(12)
#endif
#undef QK_BOYS_CASE
        default: break;
    }
    QK_CUDA_TRY(e);
    QK_CUDA_TRY(cudaMemcpyAsync(F_rows, dr.p, sizeof(double) * nout, cudaMemcpyDeviceToHost, s));
    QK_CUDA_TRY(cudaMemcpyAsync(F_one, d1.p, sizeof(double) * nout, cudaMemcpyDeviceToHost, s));
    QK_CUDA_TRY(cudaStreamSynchronize(s));
    return QK_OK;
}

// ------------------------------------------------------------- drop-in layer
void gpu_new_(int* ierr) {
    g_last_status = QK_OK;   // a new drop-in session reports only its own failures
    qk_ctx* c = qk_default_ctx();
    if (ierr) *ierr = c ? 0 : QK_ERR_NO_DEVICE;
}

void gpu_set_device_(int* gpuid, int* ierr) {
    std::lock_guard<std::mutex> g(g_default_mu);
    int ndev = 0;
    cudaGetDeviceCount(&ndev);
    if (!gpuid || *gpuid < 0 || *gpuid >= ndev) {
        if (ierr) *ierr = QK_ERR_NO_DEVICE;
        return;
    }
    g_default_device = *gpuid;
    if (ierr) *ierr = 0;
}

void gpu_init_device_(int* ierr) {
    qk_ctx* c = qk_default_ctx();
    if (ierr) *ierr = c ? 0 : QK_ERR_NO_DEVICE;
}

void gpu_allocate_scratch_(bool*) {}
void gpu_deallocate_scratch_(bool*) {}

void gpu_setup_(int* natom, int* nbasis, int*, int*, int*, int*) {
    qk_ctx* c = qk_default_ctx();
    if (!c) { fail(QK_ERR_NO_DEVICE, "gpu_setup_"); return; }
    c->natom = *natom;
    c->nbasis = *nbasis;
}

void gpu_upload_method_(int* method, bool*, double*) {
    // closed and open shell (gpu_get_cshell_eri_ / gpu_get_oshell_eri_) with HF exchange
    if (!method || *method != 0) fail(QK_ERR_UNSUPPORTED, "only HF exchange (method 0) is implemented");
}

void gpu_upload_xyz_(double* atom_xyz) {
    qk_ctx* c = qk_default_ctx();
    if (!c || !atom_xyz) { fail(QK_ERR_INVALID_ARG, "gpu_upload_xyz_"); return; }
    c->xyz.assign(atom_xyz, atom_xyz + 3 * c->natom);
}

void gpu_upload_atom_and_chg_(int*, double*) {}

void gpu_upload_basis_(int* nshell, int*, int*, int* jbasis, int*, int*, int*, double*, double*, int*,
                       int*, int*, int*, int*, int* kstart, int* katom, int*, int* kprim, int*,
                       int* Ksumtype, int*, int* Qstart, int* Qfinal, int* Qsbasis, int* Qfbasis,
                       double* gccoeff, double* cons, double* gcexpo, int* KLMN) {
    qk_ctx* c = qk_default_ctx();
    if (!c) { fail(QK_ERR_NO_DEVICE, "gpu_upload_basis_"); return; }
    std::vector<double> xyz = c->xyz;
    qk_set_basis(c, c->natom, xyz.data(), *nshell, c->nbasis, *jbasis, kstart, katom, kprim, Ksumtype,
                 Qstart, Qfinal, Qsbasis, Qfbasis, gccoeff, cons, gcexpo, KLMN, c->maxprim);
}

void gpu_upload_cutoff_matrix_(double* YCutoff, double* cutPrim) {
    qk_ctx* c = qk_default_ctx();
    if (c) qk_set_schwarz(c, YCutoff, cutPrim);
}

void gpu_upload_calculated_(double*, double*, double*, double* dense) {
    qk_ctx* c = qk_default_ctx();
    if (!c || !dense) { fail(QK_ERR_INVALID_ARG, "gpu_upload_calculated_"); return; }
    c->host_D.assign(dense, dense + (size_t)c->nbasis * c->nbasis);
    c->have_D = true;
}

void gpu_upload_cutoff_(double* cutMatrix, double* integralCutoff, double* primLimit, double*, double*) {
    qk_ctx* c = qk_default_ctx();
    if (!c || !cutMatrix || !integralCutoff || !primLimit) { fail(QK_ERR_INVALID_ARG, "gpu_upload_cutoff_"); return; }
    c->host_cutmat.assign(cutMatrix, cutMatrix + (size_t)c->nshell * c->nshell);
    c->have_cutmat = true;
    qk_set_cutoffs(c, *integralCutoff, *primLimit);
}

void gpu_get_cshell_eri_(bool*, double* o) {
    qk_ctx* c = qk_default_ctx();
    if (!c || !o) { fail(QK_ERR_INVALID_ARG, "gpu_get_cshell_eri_"); return; }
    if (!c->have_D) { fail(QK_ERR_NOT_READY, "gpu_get_cshell_eri_: density not uploaded"); return; }
    // the density (or delta density when deltaO) arrives through gpu_upload_calculated_,
    // exactly as in the reference; deltaO only changes what the caller uploaded
    qk_fock2e_host(c, c->host_D.data(), c->have_cutmat ? c->host_cutmat.data() : nullptr, o);
}

void gpu_upload_calculated_beta_(double*, double* denseb) {
    qk_ctx* c = qk_default_ctx();
    if (!c || !denseb) { fail(QK_ERR_INVALID_ARG, "gpu_upload_calculated_beta_"); return; }
    c->host_Db.assign(denseb, denseb + (size_t)c->nbasis * c->nbasis);
    c->have_Db = true;
}

void gpu_get_oshell_eri_(bool*, double* o, double* ob) {
    qk_ctx* c = qk_default_ctx();
    if (!c || !o || !ob) { fail(QK_ERR_INVALID_ARG, "gpu_get_oshell_eri_"); return; }
    if (!c->have_D || !c->have_Db) { fail(QK_ERR_NOT_READY, "gpu_get_oshell_eri_: densities not uploaded"); return; }
    qk_fock2e_uhf_host(c, c->host_D.data(), c->host_Db.data(), c->have_cutmat ? c->host_cutmat.data() : nullptr, o, ob);
}

void gpu_delete_(int* ierr) {
    std::lock_guard<std::mutex> g(g_default_mu);
    qk_destroy(g_default);
    g_default = nullptr;
    if (ierr) *ierr = 0;
}

}  // extern "C"

#endif  // QK_LANE_SP_TU
