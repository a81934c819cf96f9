// Shared constants, recursion geometry and the Boys function of the CUDA library.
#pragma once
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#ifndef QK_MAX_L
#define QK_MAX_L 2
#endif

namespace qk {

constexpr int kMaxL = QK_MAX_L;                         // compiled shell angular momentum
constexpr double kFixedScale = 17592186044416.0;        // 2^44
constexpr double kFixedInv = 1.0 / 17592186044416.0;
constexpr double kX0 = 34.986836655249725;              // 2 pi^(5/2)
constexpr double kHalfSqrtPi = 0.8862269254527579;      // sqrt(pi)/2
constexpr double kBoysDT = 0.05;
constexpr double kBoysInvDT = 20.0;
constexpr int kBoysNT = 721;                            // T in [0, 36]
constexpr int kBoysNM = 4 * kMaxL + 8;                  // m = 0 .. 4L + 7
constexpr double kBoysTmax = 36.0;
constexpr int kWarpsPerBlock = 4;

template <typename R>
struct VrrGeom {
    R PA[3], WP[3], QC[3], WQ[3];
    R oo2z, oo2e, oo2ze, rho_z, rho_e;
};

// F_0..F_M at T, each multiplied by `scale`.
template <int M>
__device__ __forceinline__ void boys_scaled(double T, double scale, const double* __restrict__ tab, double* F) {
    if (T < kBoysTmax) {
        const int k = __double2int_rn(T * kBoysInvDT);
        const double u = k * kBoysDT - T;   // -(T - T_k)
        const double* t = tab + k * kBoysNM + M;
        // 7-term Taylor expansion of F_M around T_k (|u| <= 0.025)
        double f = __ldg(t + 6) * (1.0 / 720.0);
        f = fma(f, u, __ldg(t + 5) * (1.0 / 120.0));
        f = fma(f, u, __ldg(t + 4) * (1.0 / 24.0));
        f = fma(f, u, __ldg(t + 3) * (1.0 / 6.0));
        f = fma(f, u, __ldg(t + 2) * 0.5);
        f = fma(f, u, __ldg(t + 1));
        f = fma(f, u, __ldg(t + 0));
        if (M == 0) {
            F[0] = f * scale;
        } else {
            // exp(-T) = exp(-T_k) * exp(u), exp(u) by its 7-term series (|u| <= 0.025)
            double eu = fma(u, 1.0 / 720.0, 1.0 / 120.0);
            eu = fma(eu, u, 1.0 / 24.0);
            eu = fma(eu, u, 1.0 / 6.0);
            eu = fma(eu, u, 0.5);
            eu = fma(eu, u, 1.0);
            eu = fma(eu, u, 1.0);
            const double e = __ldg(tab + kBoysNT * kBoysNM + k) * eu;
            const double T2 = 2.0 * T;
            double fm = f;
            F[M] = fm * scale;
#pragma unroll
            for (int m = M; m > 0; --m) {
                fm = fma(T2, fm, e) * (1.0 / (2 * m - 1));
                F[m - 1] = fm * scale;
            }
        }
    } else {
        double f0 = kHalfSqrtPi * rsqrt(T);
        F[0] = f0 * scale;
        if (M > 0) {
            const double e = exp(-T);
            const double h = 0.5 / T;
            double fm = f0;
#pragma unroll
            for (int m = 0; m < M; ++m) {
                fm = fma((double)(2 * m + 1), fm, -e) * h;
                F[m + 1] = fm * scale;
            }
        }
    }
}

// Boys table F_m(k * dT), m < kBoysNM, from the convergent series
// F_m(T) = exp(-T) sum_k (2T)^k / ((2m+1)(2m+3)...(2m+2k+1)) in long double.
// F_0..F_M at T from a per-M row table (kBoysNT rows of 8 doubles: F_M..F_{M+6}
// at T_k, then exp(-T_k)): the same arithmetic as boys_scaled, with four 16-byte
// loads of one 64-byte row per evaluation instead of eight 8-byte ones.
constexpr int kBoysRow = 8;
template <int M>
__device__ __forceinline__ void boys_scaled_rows(double T, double scale, const double2* __restrict__ rows,
                                                 double* F) {
    if (T < kBoysTmax) {
        const int k = __double2int_rn(T * kBoysInvDT);
        const double u = k * kBoysDT - T;
        const double2* r = rows + k * (kBoysRow / 2);
        const double2 c01 = __ldg(r), c23 = __ldg(r + 1), c45 = __ldg(r + 2), c6e = __ldg(r + 3);
        double f = c6e.x * (1.0 / 720.0);
        f = fma(f, u, c45.y * (1.0 / 120.0));
        f = fma(f, u, c45.x * (1.0 / 24.0));
        f = fma(f, u, c23.y * (1.0 / 6.0));
        f = fma(f, u, c23.x * 0.5);
        f = fma(f, u, c01.y);
        f = fma(f, u, c01.x);
        if (M == 0) {
            F[0] = f * scale;
        } else {
            double eu = fma(u, 1.0 / 720.0, 1.0 / 120.0);
            eu = fma(eu, u, 1.0 / 24.0);
            eu = fma(eu, u, 1.0 / 6.0);
            eu = fma(eu, u, 0.5);
            eu = fma(eu, u, 1.0);
            eu = fma(eu, u, 1.0);
            const double e = c6e.y * eu;
            const double T2 = 2.0 * T;
            double fm = f;
            F[M] = fm * scale;
#pragma unroll
            for (int m = M; m > 0; --m) {
                fm = fma(T2, fm, e) * (1.0 / (2 * m - 1));
                F[m - 1] = fm * scale;
            }
        }
    } else {
        double f0 = kHalfSqrtPi * rsqrt(T);
        F[0] = f0 * scale;
        if (M > 0) {
            const double e = exp(-T);
            const double h = 0.5 / T;
            double fm = f0;
#pragma unroll
            for (int m = 0; m < M; ++m) {
                fm = fma((double)(2 * m + 1), fm, -e) * h;
                F[m + 1] = fm * scale;
            }
        }
    }
}

// Row tables for M = 0 .. 4 kMaxL from boys_table(): block M holds kBoysNT rows
// of kBoysRow doubles (F_M..F_{M+6}, exp(-T_k)).
inline std::vector<double> boys_row_tables(const std::vector<double>& tab) {
    const int nM = 4 * kMaxL + 1;
    std::vector<double> r((size_t)nM * kBoysNT * kBoysRow);
    for (int M = 0; M < nM; ++M)
        for (int k = 0; k < kBoysNT; ++k) {
            double* row = &r[((size_t)M * kBoysNT + k) * kBoysRow];
            for (int j = 0; j < 7; ++j) row[j] = tab[(size_t)k * kBoysNM + M + j];
            row[7] = tab[(size_t)kBoysNT * kBoysNM + k];
        }
    return r;
}

inline std::vector<double> boys_table() {
    std::vector<double> t((size_t)kBoysNT * kBoysNM);
    for (int k = 0; k < kBoysNT; ++k) {
        long double T = (long double)k * kBoysDT;
        for (int m = 0; m < kBoysNM; ++m) {
            long double term = 1.0L / (2 * m + 1), sum = term;
            for (int j = 1; j < 4000; ++j) {
                term *= 2.0L * T / (2 * m + 2 * j + 1);
                sum += term;
                if (term < sum * 1e-22L) break;
            }
            t[(size_t)k * kBoysNM + m] = (double)(expl(-T) * sum);
        }
    }
    // exp(-T_k) after the table (used for the downward recursion)
    for (int k = 0; k < kBoysNT; ++k) t.push_back((double)expl(-(long double)k * kBoysDT));
    return t;
}

}  // namespace qk
