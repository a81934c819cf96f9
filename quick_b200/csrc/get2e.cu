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
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

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
    const int* __restrict__ pr_qa;       // per pair
    const int* __restrict__ pr_qb;
    const int* __restrict__ pr_pp0;
    const int* __restrict__ pr_npp;
    const double* __restrict__ pr_Y;
    const double* __restrict__ pp_zeta;  // per primitive pair
    const double* __restrict__ pp_oo2z;
    const double* __restrict__ pp_K;
    const double* __restrict__ pp_cut;
    const double* __restrict__ pp_P;     // 3 per primitive pair
    const double* __restrict__ pp_PA;    // 3 per primitive pair (P - centre of first shell)
    const double* __restrict__ boys;     // kBoysNT x kBoysNM
    const double* __restrict__ D;        // nbasis^2
    const double* __restrict__ cutmat;   // nshell^2
    unsigned long long* __restrict__ A;  // nbasis^2 fixed point
    unsigned long long* stats;           // optional: [quartets computed, primitive quartets computed]
    double cut, primLimit;
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
// acc[f*NE + e]; prim_screen applies QUICK's primitive cutoff.
template <int La, int Lb, int Lc, int Ld>
__device__ __forceinline__ void contract_quartet(const DevData& d, int bp0, int bnp, int kp0, int knp,
                                                 const double C[3], double dnmax, bool prim_screen,
                                                 double* acc, int* nprim_done) {
    using Cls = EriClass<La, Lb, Lc, Ld>;
    constexpr int M = Cls::M;
#pragma unroll
    for (int i = 0; i < Cls::NE * Cls::NF; ++i) acc[i] = 0.0;
    for (int i = 0; i < bnp; ++i) {
        const int pi = bp0 + i;
        const double zeta = __ldg(d.pp_zeta + pi);
        const double oo2z = __ldg(d.pp_oo2z + pi);
        const double Kab = __ldg(d.pp_K + pi) * kX0;
        const double cut1 = dnmax * __ldg(d.pp_cut + pi);
        const double Px = __ldg(d.pp_P + 3 * pi), Py = __ldg(d.pp_P + 3 * pi + 1), Pz = __ldg(d.pp_P + 3 * pi + 2);
        const double PAx = __ldg(d.pp_PA + 3 * pi), PAy = __ldg(d.pp_PA + 3 * pi + 1), PAz = __ldg(d.pp_PA + 3 * pi + 2);
        for (int j = 0; j < knp; ++j) {
            const int pj = kp0 + j;
            if (prim_screen && !(cut1 * __ldg(d.pp_cut + pj) > d.primLimit)) continue;
            ++*nprim_done;
            const double eta = __ldg(d.pp_zeta + pj);
            const double Qx = __ldg(d.pp_P + 3 * pj), Qy = __ldg(d.pp_P + 3 * pj + 1), Qz = __ldg(d.pp_P + 3 * pj + 2);
            const double s = zeta + eta;
            const double inv_s = 1.0 / s;
            const double rho_z = eta * inv_s, rho_e = zeta * inv_s;
            const double rho = zeta * rho_z;
            const double PQx = Px - Qx, PQy = Py - Qy, PQz = Pz - Qz;
            const double T = rho * (PQx * PQx + PQy * PQy + PQz * PQz);
            const double pref = Kab * __ldg(d.pp_K + pj) * sqrt(inv_s);
            double F[M + 1];
            boys_scaled<M>(T, pref, d.boys, F);
            VrrGeom<double> G;
            G.PA[0] = PAx; G.PA[1] = PAy; G.PA[2] = PAz;
            G.WP[0] = -rho_z * PQx; G.WP[1] = -rho_z * PQy; G.WP[2] = -rho_z * PQz;
            G.QC[0] = Qx - C[0]; G.QC[1] = Qy - C[1]; G.QC[2] = Qz - C[2];
            G.WQ[0] = rho_e * PQx; G.WQ[1] = rho_e * PQy; G.WQ[2] = rho_e * PQz;
            G.oo2z = oo2z;
            G.oo2e = __ldg(d.pp_oo2z + pj);
            G.oo2ze = 0.5 * inv_s;
            G.rho_z = rho_z;
            G.rho_e = rho_e;
            Cls::template vrr<double>(F, G, acc);
        }
    }
}

// One quartet (bra pair P, ket pair Q): integrals, J/K digestion.
// Lane-private updates go straight to A; the bra J block is returned in jab
// (already weighted) for the warp reduction.
template <int La, int Lb, int Lc, int Ld>
__device__ __forceinline__ void fock_quartet(const DevData& d, int P, int Q, double* jab_out, int* nq_done,
                                             int* np_done) {
    using Cls = EriClass<La, Lb, Lc, Ld>;
    constexpr int NA = Cls::NA, NB = Cls::NB, NC = Cls::NC, ND = Cls::ND;
    constexpr int NE = Cls::NE, NF = Cls::NF, NAB = NA * NB;
    const int n = d.nbasis, ns = d.nshell;
    const int qa = d.pr_qa[P], qb = d.pr_qb[P], qc = d.pr_qa[Q], qd = d.pr_qb[Q];
    const int sa = d.q_parent[qa], sb = d.q_parent[qb], sc = d.q_parent[qc], sd = d.q_parent[qd];
    const double* cm = d.cutmat;
    double dnmax = fmax(4.0 * cm[sa * ns + sb], 4.0 * cm[sc * ns + sd]);
    dnmax = fmax(dnmax, fmax(cm[sa * ns + sd], cm[sa * ns + sc]));
    dnmax = fmax(dnmax, fmax(cm[sb * ns + sc], cm[sb * ns + sd]));
    const double ct = d.pr_Y[P] * d.pr_Y[Q];
    if (!(ct * dnmax > d.cut)) return;
    ++*nq_done;

    const int ia = d.q_atom[qa], ib = d.q_atom[qb], ic = d.q_atom[qc], id = d.q_atom[qd];
    const double AB[3] = {d.xyz[3 * ia] - d.xyz[3 * ib], d.xyz[3 * ia + 1] - d.xyz[3 * ib + 1],
                          d.xyz[3 * ia + 2] - d.xyz[3 * ib + 2]};
    const double Cc[3] = {d.xyz[3 * ic], d.xyz[3 * ic + 1], d.xyz[3 * ic + 2]};
    const double CD[3] = {Cc[0] - d.xyz[3 * id], Cc[1] - d.xyz[3 * id + 1], Cc[2] - d.xyz[3 * id + 2]};

    double acc[NE * NF];
    contract_quartet<La, Lb, Lc, Ld>(d, d.pr_pp0[P], d.pr_npp[P], d.pr_pp0[Q], d.pr_npp[Q], Cc, dnmax, true, acc,
                                     np_done);

    // bra HRR per ket column
    double t1[NF * NAB];
#pragma unroll
    for (int f = 0; f < NF; ++f) Cls::hrr_bra(acc + f * NE, t1 + f * NAB, AB[0], AB[1], AB[2]);

    const int fa = d.q_f0[qa], fb = d.q_f0[qb], fc = d.q_f0[qc], fd = d.q_f0[qd];
    // degeneracy of the unique quartet (pairs are unordered, bra/ket unordered)
    const double deg = (qa != qb ? 2.0 : 1.0) * (qc != qd ? 2.0 : 1.0) * (P != Q ? 2.0 : 1.0);
    const double wJ = 0.25 * deg;      // 2 * deg/8
    const double wK = -0.0625 * deg;   // -1/2 * deg/8

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
#pragma unroll
    for (int c = 0; c < NC; ++c)
#pragma unroll
        for (int e = 0; e < ND; ++e) atomic_fixed(A + (size_t)(fc + c) * n + fd + e, wJ * jcd[c * ND + e]);
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

// Work item: x = bra pair, y = first ket pair, z = number of kets (<= 32).
template <int La, int Lb, int Lc, int Ld>
__global__ void __launch_bounds__(32 * kWarpsPerBlock)
fock_class_kernel(DevData d, const int4* __restrict__ items, int n_items, int* __restrict__ counter) {
    using Cls = EriClass<La, Lb, Lc, Ld>;
    constexpr int NAB = Cls::NA * Cls::NB;
    const int lane = threadIdx.x & 31;
    for (;;) {
        int it = 0;
        if (lane == 0) it = atomicAdd(counter, 1);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= n_items) break;
        const int4 w = items[it];
        double jab[NAB];
#pragma unroll
        for (int i = 0; i < NAB; ++i) jab[i] = 0.0;
        int nq = 0, np = 0;
        if (lane < w.z) fock_quartet<La, Lb, Lc, Ld>(d, w.x, w.y + lane, jab, &nq, &np);
        if (d.stats) {
            const unsigned sq = __reduce_add_sync(0xffffffffu, (unsigned)nq);
            const unsigned sp = __reduce_add_sync(0xffffffffu, (unsigned)np);
            if (lane == 0) {
                atomicAdd(d.stats, (unsigned long long)sq);
                atomicAdd(d.stats + 1, (unsigned long long)sp);
            }
        }
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
    if (mode >= 0) { p0 += mode; np = 1; }
    double acc[NE * NF];
    int ndone = 0;
    contract_quartet<La, Lb, La, Lb>(d, p0, np, p0, np, Cc, 0.0, false, acc, &ndone);
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

#define QK_PAIR_CLASSES(X) X(0, 0) X(1, 0) X(1, 1) X(2, 0) X(2, 1) X(2, 2)

template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0, cap = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { if (p) cudaFree(p); }
    cudaError_t reserve(size_t count) {
        n = count;
        if (count <= cap && p) return cudaSuccess;
        if (p) { cudaFree(p); p = nullptr; cap = 0; }
        if (count == 0) return cudaSuccess;
        cudaError_t e = cudaMalloc(&p, count * sizeof(T));
        if (e == cudaSuccess) cap = count;
        return e;
    }
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

struct PairTable {
    std::vector<int> qa, qb, pp0, npp;
    std::vector<double> Y;
    std::vector<double> zeta, oo2z, K, cut, P, PA;
    std::vector<Bucket> buckets;
    DevBuf<int> d_qa, d_qb, d_pp0, d_npp;
    DevBuf<double> d_Y, d_zeta, d_oo2z, d_K, d_cut, d_P, d_PA;
    void clear() {
        qa.clear(); qb.clear(); pp0.clear(); npp.clear(); Y.clear();
        zeta.clear(); oo2z.clear(); K.clear(); cut.clear(); P.clear(); PA.clear(); buckets.clear();
    }
};

using FockFn = void (*)(dim3, dim3, cudaStream_t, const DevData&, const int4*, int, int*);
template <int a, int b, int c, int e>
void launch_fock(dim3 g, dim3 bl, cudaStream_t s, const DevData& dd, const int4* it, int n, int* cnt) {
    fock_class_kernel<a, b, c, e><<<g, bl, 0, s>>>(dd, it, n, cnt);
}
template <int a, int b, int c, int e>
const void* fock_fn_ptr() { return (const void*)&fock_class_kernel<a, b, c, e>; }

struct ClassEntry {
    int La, Lb, Lc, Ld;
    FockFn fn;
    const void* (*kernel)();
    double prim_flops, quartet_flops;   // algorithmic FP64 operations (gen_eri.py model)
};
#define QK_X(a, b, c, e) {a, b, c, e, &launch_fock<a, b, c, e>, &fock_fn_ptr<a, b, c, e>, \
                          EriClass<a, b, c, e>::PRIM_FLOPS, EriClass<a, b, c, e>::QUARTET_FLOPS},
static const ClassEntry g_classes[] = {QK_ERI_CLASS_LIST(QK_X)};
#undef QK_X
constexpr int kNumClasses = sizeof(g_classes) / sizeof(g_classes[0]);

struct ClassWork {
    std::vector<int4> items;
    DevBuf<int4> d_items;
    long long nquart = 0, nprimq = 0;
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
    std::vector<int> shell_f0, shell_f1, shell_prim0;
    bool have_basis = false, have_schwarz = false;
    std::vector<double> Ycut, cutprim;   // nshell^2, jbasis^2 (symmetric)
    double integralCutoff = 1e-7, primLimit = 1e-8;
    double built_cut = -1.0;
    bool pairs_dirty = true;
    qk::PairTable pairs;
    qk::ClassWork work[qk::kNumClasses];
    int launches = 0;
    long long last_quart = 0, last_primq = 0;
    int num_sms = 148;
    // device buffers
    qk::DevBuf<double> d_xyz, d_boys, d_D, d_cutmat, d_o;
    qk::DevBuf<int> d_q_atom, d_q_f0, d_q_parent, d_q_prim0, d_q_nprim, d_shell_f0, d_shell_f1;
    qk::DevBuf<unsigned long long> d_A;
    qk::DevBuf<int> d_counters;
    // optional per-class timing (CUDA events on the launching stream) and work counters
    bool profile_events = false, profile_stats = false;
    cudaEvent_t ev[2 * qk::kNumClasses] = {};
    bool ev_recorded[qk::kNumClasses] = {};
    qk::DevBuf<unsigned long long> d_stats;
    // drop-in (reference-shaped) state
    std::vector<double> host_D, host_cutmat;
    bool have_D = false, have_cutmat = false;
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
    d.pr_qa = c->pairs.d_qa.p;
    d.pr_qb = c->pairs.d_qb.p;
    d.pr_pp0 = c->pairs.d_pp0.p;
    d.pr_npp = c->pairs.d_npp.p;
    d.pr_Y = c->pairs.d_Y.p;
    d.pp_zeta = c->pairs.d_zeta.p;
    d.pp_oo2z = c->pairs.d_oo2z.p;
    d.pp_K = c->pairs.d_K.p;
    d.pp_cut = c->pairs.d_cut.p;
    d.pp_P = c->pairs.d_P.p;
    d.pp_PA = c->pairs.d_PA.p;
    d.boys = c->d_boys.p;
    d.cut = c->integralCutoff;
    d.primLimit = c->primLimit;
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
        T.pp0.push_back((int)T.zeta.size());
        T.npp.push_back(a.nprim * b.nprim);
        const double* A = &c->xyz[3 * a.atom];
        const double* B = &c->xyz[3 * b.atom];
        const double r2 = (A[0] - B[0]) * (A[0] - B[0]) + (A[1] - B[1]) * (A[1] - B[1]) + (A[2] - B[2]) * (A[2] - B[2]);
        for (int i = 0; i < a.nprim; ++i)
            for (int j = 0; j < b.nprim; ++j) {
                const double ea = a.expo[i], eb = b.expo[j], z = ea + eb;
                // Xcoeff without X0 (src/modules/include/eri.fh:118-140)
                const double Kab = std::exp(-ea * eb / z * r2) / z * a.coef[i] * b.coef[j];
                double cp = 0.0;
                if (screened) cp = c->cutprim[(size_t)(a.prim0 + i) * c->jbasis + (b.prim0 + j)];
                T.zeta.push_back(z);
                T.oo2z.push_back(0.5 / z);
                T.K.push_back(Kab);
                T.cut.push_back(cp);
                for (int x = 0; x < 3; ++x) {
                    const double Px = (A[x] * ea + B[x] * eb) / z;
                    T.P.push_back(Px);
                    T.PA.push_back(Px - A[x]);
                }
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
    QK_CUDA_TRY(T.d_Y.upload(T.Y, s));
    QK_CUDA_TRY(T.d_zeta.upload(T.zeta, s));
    QK_CUDA_TRY(T.d_oo2z.upload(T.oo2z, s));
    QK_CUDA_TRY(T.d_K.upload(T.K, s));
    QK_CUDA_TRY(T.d_cut.upload(T.cut, s));
    QK_CUDA_TRY(T.d_P.upload(T.P, s));
    QK_CUDA_TRY(T.d_PA.upload(T.PA, s));
    return QK_OK;
}

// Work items of every class: (bra pair, first ket, count) chunks of <= 32
// kets that pass the Schwarz test, unique quartets only.
static int build_work(qk_ctx* c) {
    PairTable& T = c->pairs;
    const double cut = c->integralCutoff;
    c->launches = 0;
    for (int ci = 0; ci < kNumClasses; ++ci) {
        const ClassEntry& ce = g_classes[ci];
        ClassWork& W = c->work[ci];
        W.items.clear();
        W.nquart = W.nprimq = 0;
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
                    for (int s = 0; s < nk; s += 32)
                        tmp.push_back({make_int4(P, K.begin + s, std::min(32, nk - s), 0), cost});
                }
            }
        }
        std::stable_sort(tmp.begin(), tmp.end(), [](const Tmp& x, const Tmp& y) { return x.cost > y.cost; });
        W.items.resize(tmp.size());
        for (size_t i = 0; i < tmp.size(); ++i) W.items[i] = tmp[i].it;
        QK_CUDA_TRY(W.d_items.upload(W.items, c->stream));
        if (!W.items.empty()) {
            int bps = 0;
            QK_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, ce.kernel(), 32 * kWarpsPerBlock, 0));
            bps = std::max(bps, 1);
            const long long need = ((long long)W.items.size() + kWarpsPerBlock - 1) / kWarpsPerBlock;
            W.grid = (int)std::min<long long>((long long)bps * c->num_sms, need);
            c->launches++;
        }
    }
    c->launches += 1;  // finalize
    return QK_OK;
}

static int ensure_pairs(qk_ctx* c) {
    if (!c->have_basis) return fail(QK_ERR_NOT_READY, "basis not uploaded");
    if (!c->have_schwarz) return fail(QK_ERR_NOT_READY, "Schwarz bounds not set");
    if (!c->pairs_dirty && c->built_cut == c->integralCutoff) return QK_OK;
    build_pairs(c, true);
    int st = upload_pairs(c);
    if (st) return st;
    st = build_work(c);
    if (st) return st;
    // tables were uploaded on the context stream; builds may run on another stream
    QK_CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->built_cut = c->integralCutoff;
    c->pairs_dirty = false;
    return QK_OK;
}

static int fock2e_device(qk_ctx* c, const double* D, const double* cutmat, double* o, cudaStream_t s) {
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
    QK_CUDA_TRY(c->d_A.reserve((size_t)n * n));
    QK_CUDA_TRY(c->d_counters.reserve(kNumClasses));
    QK_CUDA_TRY(cudaMemsetAsync(c->d_A.p, 0, sizeof(unsigned long long) * n * n, s));
    QK_CUDA_TRY(cudaMemsetAsync(c->d_counters.p, 0, sizeof(int) * kNumClasses, s));
    DevData d = make_devdata(c);
    d.D = D;
    d.cutmat = cutmat;
    d.A = c->d_A.p;
    d.stats = nullptr;
    if (c->profile_stats) {
        QK_CUDA_TRY(c->d_stats.reserve(2 * kNumClasses));
        QK_CUDA_TRY(cudaMemsetAsync(c->d_stats.p, 0, sizeof(unsigned long long) * 2 * kNumClasses, s));
    }
    long long nq = 0, npq = 0;
    for (int ci = 0; ci < kNumClasses; ++ci) {
        ClassWork& W = c->work[ci];
        c->ev_recorded[ci] = false;
        if (W.items.empty()) continue;
        if (c->profile_stats) d.stats = c->d_stats.p + 2 * ci;
        if (c->profile_events) QK_CUDA_TRY(cudaEventRecord(c->ev[2 * ci], s));
        g_classes[ci].fn(dim3(W.grid), dim3(32 * kWarpsPerBlock), s, d, W.d_items.p, (int)W.items.size(),
                         c->d_counters.p + ci);
        QK_CUDA_TRY(cudaGetLastError());
        if (c->profile_events) {
            QK_CUDA_TRY(cudaEventRecord(c->ev[2 * ci + 1], s));
            c->ev_recorded[ci] = true;
        }
        nq += W.nquart;
        npq += W.nprimq;
    }
    finalize_kernel<<<(n * n + 255) / 256, 256, 0, s>>>(c->d_A.p, n, o);
    QK_CUDA_TRY(cudaGetLastError());
    c->last_quart = nq;
    c->last_primq = npq;
    return QK_OK;
}

}  // namespace qk

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
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        if (status) *status = fail(QK_ERR_CUDA, "stream creation failed");
        return nullptr;
    }
    std::vector<double> tab = boys_table();
    if (c->d_boys.upload(tab, c->stream) != cudaSuccess || cudaStreamSynchronize(c->stream) != cudaSuccess) {
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
    std::vector<int> q_atom, q_f0, q_parent, q_prim0, q_nprim;
    for (auto& q : c->qsh) {
        q_atom.push_back(q.atom); q_f0.push_back(q.f0); q_parent.push_back(q.parent);
        q_prim0.push_back(q.prim0); q_nprim.push_back(q.nprim);
    }
    cudaStream_t s = c->stream;
    QK_CUDA_TRY(c->d_xyz.upload(c->xyz, s));
    QK_CUDA_TRY(c->d_q_atom.upload(q_atom, s));
    QK_CUDA_TRY(c->d_q_f0.upload(q_f0, s));
    QK_CUDA_TRY(c->d_q_parent.upload(q_parent, s));
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
        DevBuf<unsigned long long> dY, dcp;
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
        std::vector<DevBuf<int2>> dwl(wl.size());
#define QK_SCHWARZ(a, b)                                                                          \
        {                                                                                         \
            auto& v = wl[a * (lmax + 1) + b];                                                     \
            if (!v.empty()) {                                                                     \
                auto& dv = dwl[a * (lmax + 1) + b];                                               \
                QK_CUDA_TRY(dv.upload(v, c->stream));                                             \
                schwarz_kernel<a, b><<<((int)v.size() + 127) / 128, 128, 0, c->stream>>>(         \
                    d, dv.p, (int)v.size(), c->d_q_prim0.p, c->d_q_nprim.p, ns, jb, dY.p, dcp.p); \
                QK_CUDA_TRY(cudaGetLastError());                                                  \
            }                                                                                     \
        }
        QK_PAIR_CLASSES(QK_SCHWARZ)
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
    QK_CUDA_TRY(cudaMemcpyAsync(c->d_D.p, D, sizeof(double) * n * n, cudaMemcpyHostToDevice, s));
    QK_CUDA_TRY(cudaMemsetAsync(c->d_o.p, 0, sizeof(double) * n * n, s));
    const double* cm = nullptr;
    if (cutmat) {
        QK_CUDA_TRY(c->d_cutmat.reserve((size_t)ns * ns));
        QK_CUDA_TRY(cudaMemcpyAsync(c->d_cutmat.p, cutmat, sizeof(double) * ns * ns, cudaMemcpyHostToDevice, s));
        cm = c->d_cutmat.p;
    }
    int st = fock2e_device(c, c->d_D.p, cm, c->d_o.p, s);
    if (st) return st;
    std::vector<double> G((size_t)n * n);
    QK_CUDA_TRY(cudaMemcpyAsync(G.data(), c->d_o.p, sizeof(double) * n * n, cudaMemcpyDeviceToHost, s));
    QK_CUDA_TRY(cudaStreamSynchronize(s));
    for (size_t i = 0; i < G.size(); ++i) o[i] += G[i];
    return QK_OK;
}

int qk_last_work(qk_ctx* c, long long* quartets, long long* primq, int* launches) {
    if (!c) return fail(QK_ERR_INVALID_ARG, "null context");
    if (quartets) *quartets = c->last_quart;
    if (primq) *primq = c->last_primq;
    if (launches) *launches = c->launches;
    return QK_OK;
}

int qk_launches_per_build(qk_ctx* c) { return c ? c->launches : 0; }

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

// ------------------------------------------------------------- drop-in layer
void gpu_new_(int* ierr) {
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

void gpu_upload_method_(int* method, bool* is_oshell, double*) {
    if (!method || *method != 0 || (is_oshell && *is_oshell))
        fail(QK_ERR_UNSUPPORTED, "only closed-shell HF exchange is implemented");
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

void gpu_delete_(int* ierr) {
    std::lock_guard<std::mutex> g(g_default_mu);
    qk_destroy(g_default);
    g_default = nullptr;
    if (ierr) *ierr = 0;
}

}  // extern "C"
