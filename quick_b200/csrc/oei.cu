// One-electron integrals on the device: overlap S, kinetic T and nuclear
// attraction V (nuclei plus optional external point charges, the QM/MM case).
//
// Replaces the CPU get1e path and the reference's getOEI_kernel
// (src/modules/quick_oei_module.f90:69-257, src/gpu/gpu_oei.cu:194,
// src/gpu/gpu_oei.h:193) for closed-shell SCF set-up.  Integrals use the
// McMurchie-Davidson Hermite expansion over QUICK's normalize_basis
// representation (aexp/dcoeff/itype/ncenter, src/modules/quick_basis_module.f90:385-424).
// One thread per basis-function pair (mu >= nu) and chunk of point charges;
// results are symmetric and bit-reproducible.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <mutex>
#include <vector>

#include "quick_b200.h"
#include "common.cuh"

namespace qk {

constexpr int kOeiLmax = 3;              // per function (f)
constexpr int kEj = kOeiLmax + 3;        // j up to l + 2 (kinetic)
constexpr int kEt = 2 * kOeiLmax + 3;    // t up to i + j

struct OeiArgs {
    int nbasis, maxcontract, ncharge;
    const int* ncontract;
    const int* itype;      // 3 x nbasis
    const double* aexp;    // maxcontract x nbasis
    const double* dcoeff;  // maxcontract x nbasis
    const int* ncenter;    // 1-based atom index
    const double* xyz;     // 3 x natom
    const double* cxyz;    // 3 x ncharge (nuclei first, then external charges)
    const double* cq;      // ncharge
    const double* boys;
    double *S, *T, *V;     // nbasis^2
};

// Flat index of (t, u, v) among the triples with t + u + v <= 2 * kOeiLmax,
// ordered by total degree, then t descending, then u descending.
constexpr int kTuvMax = (2 * kOeiLmax + 1) * (2 * kOeiLmax + 2) * (2 * kOeiLmax + 3) / 6;
__device__ __forceinline__ int tuv_index(int t, int u, int v) {
    const int L = t + u + v;
    const int before = L * (L + 1) * (L + 2) / 6;           // triples of lower degree
    const int r = L - t;                                     // u + v
    return before + r * (r + 1) / 2 + v;
}

// 1-D Hermite coefficients E[i][j][t], i <= li, j <= lj, for one Cartesian axis.
__device__ __forceinline__ void hermite_E(int li, int lj, double XPA, double XPB, double oo2p, double E0,
                                          double E[kOeiLmax + 1][kEj][kEt]) {
    for (int i = 0; i <= li; ++i)
        for (int j = 0; j <= lj; ++j)
            for (int t = 0; t < kEt; ++t) E[i][j][t] = 0.0;
    E[0][0][0] = E0;
    for (int i = 0; i <= li; ++i) {
        for (int j = 0; j <= lj; ++j) {
            if (i == 0 && j == 0) continue;
            for (int t = 0; t <= i + j; ++t) {
                double v;
                if (j == 0) {
                    const double a = t > 0 ? E[i - 1][0][t - 1] : 0.0;
                    const double b = t <= i - 1 ? E[i - 1][0][t] : 0.0;
                    const double c = t + 1 <= i - 1 ? E[i - 1][0][t + 1] : 0.0;
                    v = oo2p * a + XPA * b + (t + 1) * c;
                } else {
                    const int tm = i + j - 1;
                    const double a = t > 0 ? E[i][j - 1][t - 1] : 0.0;
                    const double b = t <= tm ? E[i][j - 1][t] : 0.0;
                    const double c = t + 1 <= tm ? E[i][j - 1][t + 1] : 0.0;
                    v = oo2p * a + XPB * b + (t + 1) * c;
                }
                E[i][j][t] = v;
            }
        }
    }
}

// grid (pairs / 128, charge chunks): chunk y sums the attraction of charges
// [y * chunk, (y + 1) * chunk) into Vpart[y][pair]; chunk 0 also writes S and T.
__global__ void oei_kernel(OeiArgs a, int chunk, double* __restrict__ Vpart) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = a.nbasis;
    const int npair = n * (n + 1) / 2;
    if (t >= npair) return;
    const int c0 = blockIdx.y * chunk;
    const int c1 = min(a.ncharge, c0 + chunk);
    const bool first = blockIdx.y == 0;
    // t -> (mu, nu), mu >= nu
    int mu = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
    while (mu * (mu + 1) / 2 > t) --mu;
    while ((mu + 1) * (mu + 2) / 2 <= t) ++mu;
    const int nu = t - mu * (mu + 1) / 2;
    const int la[3] = {a.itype[3 * mu], a.itype[3 * mu + 1], a.itype[3 * mu + 2]};
    const int lb[3] = {a.itype[3 * nu], a.itype[3 * nu + 1], a.itype[3 * nu + 2]};
    const double* A = a.xyz + 3 * (a.ncenter[mu] - 1);
    const double* B = a.xyz + 3 * (a.ncenter[nu] - 1);
    const int Lsum = la[0] + la[1] + la[2] + lb[0] + lb[1] + lb[2];
    double s = 0.0, tk = 0.0, v = 0.0;
    double E[3][kOeiLmax + 1][kEj][kEt];
    for (int p = 0; p < a.ncontract[mu]; ++p) {
        const double al = a.aexp[p + a.maxcontract * mu];
        const double ca = a.dcoeff[p + a.maxcontract * mu];
        for (int q = 0; q < a.ncontract[nu]; ++q) {
            const double be = a.aexp[q + a.maxcontract * nu];
            const double cb = a.dcoeff[q + a.maxcontract * nu];
            const double pz = al + be, oo2p = 0.5 / pz, mu_r = al * be / pz;
            double P[3];
            for (int x = 0; x < 3; ++x) {
                P[x] = (al * A[x] + be * B[x]) / pz;
                const double XAB = A[x] - B[x];
                hermite_E(la[x], lb[x] + 2, P[x] - A[x], P[x] - B[x], oo2p, exp(-mu_r * XAB * XAB), E[x]);
            }
            const double sq = sqrt(M_PI / pz);
            double S1[3], T1[3];
            for (int x = 0; x < 3; ++x) {
                const int i = la[x], j = lb[x];
                const double sij = E[x][i][j][0] * sq;
                const double sj2 = E[x][i][j + 2][0] * sq;
                const double sjm = j >= 2 ? E[x][i][j - 2][0] * sq : 0.0;
                S1[x] = sij;
                T1[x] = -2.0 * be * be * sj2 + be * (2 * j + 1) * sij - 0.5 * j * (j - 1) * sjm;
            }
            const double cc = ca * cb;
            s += cc * S1[0] * S1[1] * S1[2];
            tk += cc * (T1[0] * S1[1] * S1[2] + S1[0] * T1[1] * S1[2] + S1[0] * S1[1] * T1[2]);
            // nuclear attraction: (2 pi / p) sum_tuv E_t E_u E_v R_tuv, with the
            // Hermite Coulomb integrals R built level by level (k = Lsum .. 0) in
            // two flat arrays over t + u + v <= Lsum - k
            const double pref = cc * 2.0 * M_PI / pz;
            const int lx = la[0] + lb[0], ly = la[1] + lb[1], lz = la[2] + lb[2];
            double Ex[2 * kOeiLmax + 1], Ey[2 * kOeiLmax + 1], Ez[2 * kOeiLmax + 1];
            for (int q2 = 0; q2 <= 2 * kOeiLmax; ++q2) {
                Ex[q2] = q2 <= lx ? E[0][la[0]][lb[0]][q2] : 0.0;
                Ey[q2] = q2 <= ly ? E[1][la[1]][lb[1]][q2] : 0.0;
                Ez[q2] = q2 <= lz ? E[2][la[2]][lb[2]][q2] : 0.0;
            }
            double m2p[2 * kOeiLmax + 1];   // (-2p)^k
            m2p[0] = 1.0;
            for (int k = 1; k <= 2 * kOeiLmax; ++k) m2p[k] = m2p[k - 1] * (-2.0 * pz);
            for (int c = c0; c < c1; ++c) {
                const double PC[3] = {P[0] - a.cxyz[3 * c], P[1] - a.cxyz[3 * c + 1], P[2] - a.cxyz[3 * c + 2]};
                const double r2 = PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2];
                double F[2 * kOeiLmax + 1];
                boys_scaled<2 * kOeiLmax>(pz * r2, 1.0, a.boys, F);
                double Ra[kTuvMax], Rb[kTuvMax];
                double* Rn = Ra;   // level k + 1
                double* Rc = Rb;   // level k
                Rn[0] = m2p[Lsum] * F[Lsum];
                for (int k = Lsum - 1; k >= 0; --k) {
                    const int L = Lsum - k;
                    Rc[0] = m2p[k] * F[k];
                    for (int tt = 0; tt <= L; ++tt)
                        for (int uu = 0; uu <= L - tt; ++uu)
                            for (int vv = 0; vv <= L - tt - uu; ++vv) {
                                if (tt + uu + vv == 0) continue;
                                double r;
                                if (tt > 0) {
                                    r = PC[0] * Rn[tuv_index(tt - 1, uu, vv)];
                                    if (tt > 1) r += (tt - 1) * Rn[tuv_index(tt - 2, uu, vv)];
                                } else if (uu > 0) {
                                    r = PC[1] * Rn[tuv_index(tt, uu - 1, vv)];
                                    if (uu > 1) r += (uu - 1) * Rn[tuv_index(tt, uu - 2, vv)];
                                } else {
                                    r = PC[2] * Rn[tuv_index(tt, uu, vv - 1)];
                                    if (vv > 1) r += (vv - 1) * Rn[tuv_index(tt, uu, vv - 2)];
                                }
                                Rc[tuv_index(tt, uu, vv)] = r;
                            }
                    double* tmp = Rn; Rn = Rc; Rc = tmp;
                }
                // Rn holds level 0
                double vc = 0.0;
                for (int tt = 0; tt <= lx; ++tt)
                    for (int uu = 0; uu <= ly; ++uu)
                        for (int vv = 0; vv <= lz; ++vv) vc += Ex[tt] * Ey[uu] * Ez[vv] * Rn[tuv_index(tt, uu, vv)];
                v -= a.cq[c] * pref * vc;
            }
        }
    }
    if (first) {
        a.S[(size_t)mu * n + nu] = s; a.S[(size_t)nu * n + mu] = s;
        a.T[(size_t)mu * n + nu] = tk; a.T[(size_t)nu * n + mu] = tk;
    }
    Vpart[(size_t)blockIdx.y * npair + t] = v;
}

// Attraction to external point charges at the shell-pair level (shells up to d):
// per primitive pair and charge the Hermite Coulomb integrals R_tuv are built
// once and contracted with the Hermite coefficients of every Cartesian
// component pair of the two shells (the function-pair kernel rebuilds them for
// each component pair: 36 times for a d-d pair).  Components in QUICK's order
// (normalize_basis: p x, y, z; d xx, xy, yy, xz, yz, zz), checked on the host.
// Thread = (shell pair, chunk of charges); writes the chunk's partial sums of
// the shell pair's function pairs.
// exponent along `axis` of Cartesian component i of an L shell (L <= 2), QUICK's order
__host__ __device__ constexpr int cart_exp(int L, int i, int axis) {
    return L == 0 ? 0
         : L == 1 ? (i == axis ? 1 : 0)
         : axis == 0 ? (i == 0 ? 2 : (i == 1 || i == 3) ? 1 : 0)
         : axis == 1 ? (i == 2 ? 2 : (i == 1 || i == 4) ? 1 : 0)
                     : (i == 5 ? 2 : (i == 3 || i == 4) ? 1 : 0);
}

template <int LI, int LJ>
__device__ __forceinline__ void hermite_E_fixed(double XPA, double XPB, double oo2p, double E0,
                                                double (&E)[LI + 1][LJ + 1][LI + LJ + 1]) {
#pragma unroll
    for (int i = 0; i <= LI; ++i)
#pragma unroll
        for (int j = 0; j <= LJ; ++j)
#pragma unroll
            for (int t = 0; t <= LI + LJ; ++t) E[i][j][t] = 0.0;
    E[0][0][0] = E0;
#pragma unroll
    for (int i = 0; i <= LI; ++i)
#pragma unroll
        for (int j = 0; j <= LJ; ++j) {
            if (i == 0 && j == 0) continue;
#pragma unroll
            for (int t = 0; t <= i + j; ++t) {
                double v;
                if (j == 0) {
                    const double a = t > 0 ? E[i - 1][0][t - 1] : 0.0;
                    const double b = t <= i - 1 ? E[i - 1][0][t] : 0.0;
                    const double c = t + 1 <= i - 1 ? E[i - 1][0][t + 1] : 0.0;
                    v = oo2p * a + XPA * b + (t + 1) * c;
                } else {
                    const int tm = i + j - 1;
                    const double a = t > 0 ? E[i][j - 1][t - 1] : 0.0;
                    const double b = t <= tm ? E[i][j - 1][t] : 0.0;
                    const double c = t + 1 <= tm ? E[i][j - 1][t + 1] : 0.0;
                    v = oo2p * a + XPB * b + (t + 1) * c;
                }
                E[i][j][t] = v;
            }
        }
}

template <int LA, int LB>
__global__ void oei_charge_shell_kernel(OeiArgs a, const int4* __restrict__ pairs, int npairs, int c_begin, int chunk,
                                        int part0, double* __restrict__ Vpart) {
    constexpr int NA = (LA + 1) * (LA + 2) / 2, NB = (LB + 1) * (LB + 2) / 2, L = LA + LB;
    constexpr int NT = (L + 1) * (L + 2) * (L + 3) / 6;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= npairs) return;
    const int4 sp = pairs[t];   // first functions of the shells (L = LA, LB), same-shell flag
    const int fa0 = sp.x, fb0 = sp.y;
    const bool same = sp.z != 0;
    const int c0 = c_begin + blockIdx.y * chunk;
    const int c1 = min(a.ncharge, c0 + chunk);
    const int n = a.nbasis;
    const double* A = a.xyz + 3 * (a.ncenter[fa0] - 1);
    const double* B = a.xyz + 3 * (a.ncenter[fb0] - 1);
    double acc[NA * NB];
#pragma unroll
    for (int k = 0; k < NA * NB; ++k) acc[k] = 0.0;
    for (int p = 0; p < a.ncontract[fa0]; ++p) {
        const double al = a.aexp[p + a.maxcontract * fa0];
        for (int q = 0; q < a.ncontract[fb0]; ++q) {
            const double be = a.aexp[q + a.maxcontract * fb0];
            const double pz = al + be, oo2p = 0.5 / pz, mu_r = al * be / pz;
            double P[3];
            double Ex[LA + 1][LB + 1][L + 1], Ey[LA + 1][LB + 1][L + 1], Ez[LA + 1][LB + 1][L + 1];
            P[0] = (al * A[0] + be * B[0]) / pz;
            P[1] = (al * A[1] + be * B[1]) / pz;
            P[2] = (al * A[2] + be * B[2]) / pz;
            hermite_E_fixed<LA, LB>(P[0] - A[0], P[0] - B[0], oo2p, exp(-mu_r * (A[0] - B[0]) * (A[0] - B[0])), Ex);
            hermite_E_fixed<LA, LB>(P[1] - A[1], P[1] - B[1], oo2p, exp(-mu_r * (A[1] - B[1]) * (A[1] - B[1])), Ey);
            hermite_E_fixed<LA, LB>(P[2] - A[2], P[2] - B[2], oo2p, exp(-mu_r * (A[2] - B[2]) * (A[2] - B[2])), Ez);
            double cpref[NA * NB];   // c_a c_b 2 pi / p per component pair
            const double base = 2.0 * M_PI / pz;
#pragma unroll
            for (int i = 0; i < NA; ++i)
#pragma unroll
                for (int j = 0; j < NB; ++j)
                    cpref[i * NB + j] = a.dcoeff[p + a.maxcontract * (fa0 + i)] *
                                        a.dcoeff[q + a.maxcontract * (fb0 + j)] * base;
            double m2p[L + 1];
            m2p[0] = 1.0;
#pragma unroll
            for (int k = 1; k <= L; ++k) m2p[k] = m2p[k - 1] * (-2.0 * pz);
            for (int c = c0; c < c1; ++c) {
                const double PC[3] = {P[0] - a.cxyz[3 * c], P[1] - a.cxyz[3 * c + 1], P[2] - a.cxyz[3 * c + 2]};
                double F[L + 1];
                boys_scaled<L>(pz * (PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2]), 1.0, a.boys, F);
                double R[NT], Rn[NT];
                Rn[0] = m2p[L] * F[L];
#pragma unroll
                for (int k = L - 1; k >= 0; --k) {
                    const int Lk = L - k;
                    R[0] = m2p[k] * F[k];
#pragma unroll
                    for (int tt = 0; tt <= Lk; ++tt)
#pragma unroll
                        for (int uu = 0; uu <= Lk - tt; ++uu)
#pragma unroll
                            for (int vv = 0; vv <= Lk - tt - uu; ++vv) {
                                if (tt + uu + vv == 0) continue;
                                double r;
                                if (tt > 0) {
                                    r = PC[0] * Rn[tuv_index(tt - 1, uu, vv)];
                                    if (tt > 1) r += (tt - 1) * Rn[tuv_index(tt - 2, uu, vv)];
                                } else if (uu > 0) {
                                    r = PC[1] * Rn[tuv_index(tt, uu - 1, vv)];
                                    if (uu > 1) r += (uu - 1) * Rn[tuv_index(tt, uu - 2, vv)];
                                } else {
                                    r = PC[2] * Rn[tuv_index(tt, uu, vv - 1)];
                                    if (vv > 1) r += (vv - 1) * Rn[tuv_index(tt, uu, vv - 2)];
                                }
                                R[tuv_index(tt, uu, vv)] = r;
                            }
#pragma unroll
                    for (int k2 = 0; k2 < NT; ++k2) Rn[k2] = R[k2];
                }
                if (L == 0) R[0] = Rn[0];
                const double qc = a.cq[c];
#pragma unroll
                for (int i = 0; i < NA; ++i)
#pragma unroll
                    for (int j = 0; j < NB; ++j) {
                        const int ax = cart_exp(LA, i, 0), ay = cart_exp(LA, i, 1), az = cart_exp(LA, i, 2);
                        const int bx = cart_exp(LB, j, 0), by = cart_exp(LB, j, 1), bz = cart_exp(LB, j, 2);
                        const int lx = ax + bx, ly = ay + by, lz = az + bz;
                        double vc = 0.0;
#pragma unroll
                        for (int tt = 0; tt <= lx; ++tt)
#pragma unroll
                            for (int uu = 0; uu <= ly; ++uu)
#pragma unroll
                                for (int vv = 0; vv <= lz; ++vv)
                                    vc += Ex[ax][bx][tt] * Ey[ay][by][uu] * Ez[az][bz][vv] *
                                          R[tuv_index(tt, uu, vv)];
                        acc[i * NB + j] -= qc * cpref[i * NB + j] * vc;
                    }
            }
        }
    }
    const size_t npf = (size_t)n * (n + 1) / 2;
    double* out = Vpart + (size_t)(part0 + blockIdx.y) * npf;
#pragma unroll
    for (int i = 0; i < NA; ++i)
#pragma unroll
        for (int j = 0; j < NB; ++j) {
            const int f = fa0 + i, g = fb0 + j;
            if (same && f < g) continue;
            const int mu = f > g ? f : g, nu = f > g ? g : f;
            out[(size_t)mu * (mu + 1) / 2 + nu] = acc[i * NB + j];
        }
}

// V = sum of the chunks' partial sums, in chunk order (bit-reproducible).
__global__ void oei_reduce_kernel(OeiArgs a, int nchunk, const double* __restrict__ Vpart) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = a.nbasis;
    const int npair = n * (n + 1) / 2;
    if (t >= npair) return;
    int mu = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
    while (mu * (mu + 1) / 2 > t) --mu;
    while ((mu + 1) * (mu + 2) / 2 <= t) ++mu;
    const int nu = t - mu * (mu + 1) / 2;
    double v = 0.0;
    for (int k = 0; k < nchunk; ++k) v += Vpart[(size_t)k * npair + t];
    a.V[(size_t)mu * n + nu] = v;
    a.V[(size_t)nu * n + mu] = v;
}

// One non-blocking stream per device for the one-electron set-up, so that it
// neither waits for nor holds up work on other streams (no device-wide syncs:
// stream-ordered allocation, copies and a stream synchronisation only).
static cudaStream_t oei_stream(int device) {
    static std::mutex mu;
    static cudaStream_t streams[64] = {};
    std::lock_guard<std::mutex> g(mu);
    if (device < 0 || device >= 64) return nullptr;
    if (!streams[device]) {
        // highest priority, as the contexts' set-up streams (see qk_create)
        int lo = 0, hi = 0;
        cudaDeviceGetStreamPriorityRange(&lo, &hi);
        cudaStreamCreateWithPriority(&streams[device], cudaStreamNonBlocking, hi);
    }
    return streams[device];
}

static const std::vector<double>& oei_boys_table() {
    static std::once_flag once;
    static std::vector<double> tab;
    std::call_once(once, [] { tab = boys_table(); });
    return tab;
}

}  // namespace qk

extern "C" int qk_oei_host(int device, int natom, const double* xyz, const double* Z, int nbasis, int maxcontract,
                           const int* ncontract, const int* itype, const double* aexp, const double* dcoeff,
                           const int* ncenter, int next, const double* ext_xyz, const double* ext_q,
                           double* S, double* T, double* V) {
    using namespace qk;
    if (natom <= 0 || nbasis <= 0 || maxcontract <= 0 || !xyz || !Z || !ncontract || !itype || !aexp ||
        !dcoeff || !ncenter || !S || !T || !V || next < 0 || (next > 0 && (!ext_xyz || !ext_q)))
        return QK_ERR_INVALID_ARG;
    for (int i = 0; i < 3 * nbasis; ++i)
        if (itype[i] < 0 || itype[i] > kOeiLmax) return QK_ERR_UNSUPPORTED;
    for (int i = 0; i < nbasis; ++i)
        if (ncenter[i] < 1 || ncenter[i] > natom || ncontract[i] < 1 || ncontract[i] > maxcontract)
            return QK_ERR_INVALID_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return QK_ERR_CUDA;
    const int nq = natom + next;
    std::vector<double> cxyz(3 * (size_t)nq), cq(nq);
    for (int i = 0; i < natom; ++i) {
        for (int k = 0; k < 3; ++k) cxyz[3 * i + k] = xyz[3 * i + k];
        cq[i] = Z[i];
    }
    for (int i = 0; i < next; ++i) {
        for (int k = 0; k < 3; ++k) cxyz[3 * (natom + i) + k] = ext_xyz[3 * i + k];
        cq[natom + i] = ext_q[i];
    }
    const std::vector<double>& tab = oei_boys_table();
    const size_t nn = (size_t)nbasis * nbasis;
    const long long npair = (long long)nbasis * (nbasis + 1) / 2;
    // charge chunks: enough blocks for about 4 waves of the GPU, at least 32 charges a chunk
    const long long want = std::max<long long>(1, (4LL * 148 * 2048 + npair - 1) / npair);
    // external charges go to the shell-pair kernel when every shell is s, p or d in
    // QUICK's component order; the function-pair kernel takes the nuclei (and all
    // charges otherwise)
    std::vector<int4> sp_list[3][3];
    bool shells = next > 0;
    {
        const int comp[3][6][3] = {{{0, 0, 0}},
                                   {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}},
                                   {{2, 0, 0}, {1, 1, 0}, {0, 2, 0}, {1, 0, 1}, {0, 1, 1}, {0, 0, 2}}};
        std::vector<int> f0, Ls;
        for (int f = 0; f < nbasis && shells;) {
            const int L = itype[3 * f] + itype[3 * f + 1] + itype[3 * f + 2];
            if (L > 2) { shells = false; break; }
            const int nc = (L + 1) * (L + 2) / 2;
            if (f + nc > nbasis) { shells = false; break; }
            for (int k = 0; k < nc && shells; ++k) {
                const int g = f + k;
                shells = itype[3 * g] == comp[L][k][0] && itype[3 * g + 1] == comp[L][k][1] &&
                         itype[3 * g + 2] == comp[L][k][2] && ncenter[g] == ncenter[f] &&
                         ncontract[g] == ncontract[f];
                for (int p = 0; p < ncontract[f] && shells; ++p)
                    shells = aexp[p + (size_t)maxcontract * g] == aexp[p + (size_t)maxcontract * f];
            }
            f0.push_back(f);
            Ls.push_back(L);
            f += nc;
        }
        if (shells)
            for (int i = 0; i < (int)f0.size(); ++i)
                for (int j = 0; j <= i; ++j) {
                    const bool swap = Ls[j] > Ls[i];
                    const int a0 = swap ? f0[j] : f0[i], b0 = swap ? f0[i] : f0[j];
                    const int la = swap ? Ls[j] : Ls[i], lb = swap ? Ls[i] : Ls[j];
                    sp_list[la][lb].push_back(make_int4(a0, b0, i == j ? 1 : 0, 0));
                }
    }
    long long nsp = 0;
    for (auto& row : sp_list)
        for (auto& v : row) nsp += (long long)v.size();
    const int nq_fn = shells ? natom : nq;      // charges of the function-pair kernel
    const int nchunk = (int)std::max<long long>(1, std::min<long long>({want, (nq_fn + 31) / 32, 65535LL}));
    const int chunk = (nq_fn + nchunk - 1) / nchunk;
    const long long want_sp = std::max<long long>(1, (4LL * 148 * 2048 + nsp - 1) / std::max<long long>(nsp, 1));
    const int nchunk_e = shells ? (int)std::max<long long>(1, std::min<long long>({want_sp, (next + 31) / 32, 65535LL}))
                                : 0;
    const int chunk_e = shells ? (next + nchunk_e - 1) / nchunk_e : 0;
    int n_sp_lists = 0;
    for (auto& row : sp_list)
        for (auto& v : row) n_sp_lists += v.empty() ? 0 : 1;
    (void)n_sp_lists;
    cudaStream_t s = oei_stream(device);
    if (!s) return QK_ERR_CUDA;
    // one device block: inputs, then S T V, then the partial sums
    std::vector<int4> sp_all;
    size_t sp_off[3][3] = {};
    for (int la = 0; la < 3; ++la)
        for (int lb = 0; lb < 3; ++lb) {
            sp_off[la][lb] = sp_all.size();
            sp_all.insert(sp_all.end(), sp_list[la][lb].begin(), sp_list[la][lb].end());
        }
    size_t sizes[11] = {nbasis * sizeof(int), 3 * nbasis * sizeof(int), (size_t)maxcontract * nbasis * 8,
                        (size_t)maxcontract * nbasis * 8, nbasis * sizeof(int), 3 * (size_t)natom * 8,
                        cxyz.size() * 8, cq.size() * 8, tab.size() * 8, sp_all.size() * sizeof(int4), 3 * nn * 8};
    const void* src[10] = {ncontract, itype, aexp, dcoeff, ncenter, xyz, cxyz.data(), cq.data(), tab.data(),
                           sp_all.data()};
    size_t off[12];
    off[0] = 0;
    for (int i = 0; i < 11; ++i) off[i + 1] = off[i] + ((sizes[i] + 255) & ~size_t(255));
    const int nparts = nchunk + nchunk_e;
    const size_t total = off[11] + (size_t)nparts * npair * 8;
    char* base = nullptr;
    if (cudaMallocAsync((void**)&base, total, s) != cudaSuccess) return QK_ERR_OUT_OF_MEMORY;
    int st = QK_OK;
    for (int i = 0; i < 10 && st == QK_OK; ++i)
        if (sizes[i] > 0 && cudaMemcpyAsync(base + off[i], src[i], sizes[i], cudaMemcpyHostToDevice, s) != cudaSuccess)
            st = QK_ERR_CUDA;
    if (st == QK_OK) {
        OeiArgs a;
        a.nbasis = nbasis; a.maxcontract = maxcontract; a.ncharge = nq_fn;
        a.ncontract = (const int*)(base + off[0]); a.itype = (const int*)(base + off[1]);
        a.aexp = (const double*)(base + off[2]); a.dcoeff = (const double*)(base + off[3]);
        a.ncenter = (const int*)(base + off[4]); a.xyz = (const double*)(base + off[5]);
        a.cxyz = (const double*)(base + off[6]); a.cq = (const double*)(base + off[7]);
        a.boys = (const double*)(base + off[8]);
        a.S = (double*)(base + off[10]); a.T = a.S + nn; a.V = a.T + nn;
        double* Vpart = (double*)(base + off[11]);
        const int gx = (int)((npair + 127) / 128);
        oei_kernel<<<dim3(gx, nchunk), 128, 0, s>>>(a, chunk, Vpart);
        if (nchunk_e > 0) {
            OeiArgs ae = a;
            ae.ncharge = nq;
            const int4* dsp = (const int4*)(base + off[9]);
#define QK_OEI_SP(LA, LB)                                                                              \
            if (!sp_list[LA][LB].empty()) {                                                            \
                const int np_ = (int)sp_list[LA][LB].size();                                           \
                oei_charge_shell_kernel<LA, LB><<<dim3((np_ + 63) / 64, nchunk_e), 64, 0, s>>>(          \
                    ae, dsp + sp_off[LA][LB], np_, natom, chunk_e, nchunk, Vpart);                      \
            }
            QK_OEI_SP(0, 0) QK_OEI_SP(1, 0) QK_OEI_SP(1, 1) QK_OEI_SP(2, 0) QK_OEI_SP(2, 1) QK_OEI_SP(2, 2)
#undef QK_OEI_SP
        }
        oei_reduce_kernel<<<gx, 128, 0, s>>>(a, nparts, Vpart);
        if (cudaGetLastError() != cudaSuccess) st = QK_ERR_CUDA;
        if (st == QK_OK && (cudaMemcpyAsync(S, a.S, nn * 8, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                            cudaMemcpyAsync(T, a.T, nn * 8, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                            cudaMemcpyAsync(V, a.V, nn * 8, cudaMemcpyDeviceToHost, s) != cudaSuccess))
            st = QK_ERR_CUDA;
    }
    cudaFreeAsync(base, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) st = QK_ERR_CUDA;
    return st;
}
