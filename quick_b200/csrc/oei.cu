// One-electron integrals on the device: overlap S, kinetic T and nuclear
// attraction V (nuclei plus optional external point charges, the QM/MM case).
//
// Replaces the CPU get1e path and the reference's getOEI_kernel
// (src/modules/quick_oei_module.f90:69-257, src/gpu/gpu_oei.cu:194,
// src/gpu/gpu_oei.h:193) for closed-shell SCF set-up.  Integrals use the
// McMurchie-Davidson Hermite expansion over QUICK's normalize_basis
// representation (aexp/dcoeff/itype/ncenter, src/modules/quick_basis_module.f90:385-424).
// One thread per basis-function pair (mu >= nu); results are symmetric.
#include <cuda_runtime.h>

#include <cstdio>
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

__global__ void oei_kernel(OeiArgs a) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = a.nbasis;
    if (t >= n * (n + 1) / 2) return;
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
            // nuclear attraction: (2 pi / p) sum_tuv E_t E_u E_v R_tuv
            const double pref = cc * 2.0 * M_PI / pz;
            for (int c = 0; c < a.ncharge; ++c) {
                const double PC[3] = {P[0] - a.cxyz[3 * c], P[1] - a.cxyz[3 * c + 1], P[2] - a.cxyz[3 * c + 2]};
                const double r2 = PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2];
                double F[2 * kOeiLmax + 1];
                boys_scaled<2 * kOeiLmax>(pz * r2, 1.0, a.boys, F);
                // R[n][t][u][v], n + t + u + v <= Lsum
                double R[2 * kOeiLmax + 1][2 * kOeiLmax + 1][2 * kOeiLmax + 1][2 * kOeiLmax + 1];
                double m2p = 1.0;
                for (int k = 0; k <= Lsum; ++k) {
                    R[k][0][0][0] = m2p * F[k];
                    m2p *= -2.0 * pz;
                }
                for (int k = Lsum - 1; k >= 0; --k) {
                    const int L = Lsum - k;   // t+u+v <= L at level k
                    for (int tt = 0; tt <= L; ++tt)
                        for (int uu = 0; uu <= L - tt; ++uu)
                            for (int vv = 0; vv <= L - tt - uu; ++vv) {
                                if (tt + uu + vv == 0) continue;
                                double r;
                                if (tt > 0) {
                                    r = PC[0] * R[k + 1][tt - 1][uu][vv];
                                    if (tt > 1) r += (tt - 1) * R[k + 1][tt - 2][uu][vv];
                                } else if (uu > 0) {
                                    r = PC[1] * R[k + 1][tt][uu - 1][vv];
                                    if (uu > 1) r += (uu - 1) * R[k + 1][tt][uu - 2][vv];
                                } else {
                                    r = PC[2] * R[k + 1][tt][uu][vv - 1];
                                    if (vv > 1) r += (vv - 1) * R[k + 1][tt][uu][vv - 2];
                                }
                                R[k][tt][uu][vv] = r;
                            }
                }
                double vc = 0.0;
                for (int tt = 0; tt <= la[0] + lb[0]; ++tt)
                    for (int uu = 0; uu <= la[1] + lb[1]; ++uu)
                        for (int vv = 0; vv <= la[2] + lb[2]; ++vv)
                            vc += E[0][la[0]][lb[0]][tt] * E[1][la[1]][lb[1]][uu] * E[2][la[2]][lb[2]][vv] *
                                  R[0][tt][uu][vv];
                v -= a.cq[c] * pref * vc;
            }
        }
    }
    a.S[(size_t)mu * n + nu] = s; a.S[(size_t)nu * n + mu] = s;
    a.T[(size_t)mu * n + nu] = tk; a.T[(size_t)nu * n + mu] = tk;
    a.V[(size_t)mu * n + nu] = v; a.V[(size_t)nu * n + mu] = v;
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
    std::vector<double> tab = boys_table();
    const size_t nn = (size_t)nbasis * nbasis;
    void* bufs[11] = {};
    size_t sizes[11] = {nbasis * sizeof(int), 3 * nbasis * sizeof(int), (size_t)maxcontract * nbasis * 8,
                        (size_t)maxcontract * nbasis * 8, nbasis * sizeof(int), 3 * (size_t)natom * 8,
                        cxyz.size() * 8, cq.size() * 8, tab.size() * 8, 3 * nn * 8, 0};
    const void* src[10] = {ncontract, itype, aexp, dcoeff, ncenter, xyz, cxyz.data(), cq.data(), tab.data(), nullptr};
    int st = QK_OK;
    for (int i = 0; i < 10 && st == QK_OK; ++i) {
        if (cudaMalloc(&bufs[i], sizes[i]) != cudaSuccess) { st = QK_ERR_OUT_OF_MEMORY; break; }
        if (src[i] && cudaMemcpy(bufs[i], src[i], sizes[i], cudaMemcpyHostToDevice) != cudaSuccess) st = QK_ERR_CUDA;
    }
    if (st == QK_OK) {
        OeiArgs a;
        a.nbasis = nbasis; a.maxcontract = maxcontract; a.ncharge = nq;
        a.ncontract = (const int*)bufs[0]; a.itype = (const int*)bufs[1];
        a.aexp = (const double*)bufs[2]; a.dcoeff = (const double*)bufs[3];
        a.ncenter = (const int*)bufs[4]; a.xyz = (const double*)bufs[5];
        a.cxyz = (const double*)bufs[6]; a.cq = (const double*)bufs[7]; a.boys = (const double*)bufs[8];
        a.S = (double*)bufs[9]; a.T = a.S + nn; a.V = a.T + nn;
        const int npair = nbasis * (nbasis + 1) / 2;
        oei_kernel<<<(npair + 127) / 128, 128>>>(a);
        if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) st = QK_ERR_CUDA;
        if (st == QK_OK && (cudaMemcpy(S, a.S, nn * 8, cudaMemcpyDeviceToHost) != cudaSuccess ||
                            cudaMemcpy(T, a.T, nn * 8, cudaMemcpyDeviceToHost) != cudaSuccess ||
                            cudaMemcpy(V, a.V, nn * 8, cudaMemcpyDeviceToHost) != cudaSuccess))
            st = QK_ERR_CUDA;
    }
    for (int i = 0; i < 10; ++i)
        if (bufs[i]) cudaFree(bufs[i]);
    return st;
}
