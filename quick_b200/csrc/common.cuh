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

// QUICK's own Boys function (src/subs/fmt.f90:13-85; its device copy is
// src/gpu/gpu_fmt.h:5-72), for the reference-faithful mode (qk_set_boys): fitted
// polynomials in 1/X above X = 5, polynomials around X = 4 and 2 on (1, 5], a
// polynomial on (0.1, 1] (down to 1e-4 when M < 4), F_M = (1 - X)/(2M + 1) below,
// then upward recursion from F_0 or downward from F_M.  It is first order in X
// below 0.1 and its upward recursion loses precision for large M at small X (at
// M = 12, X in (0.1, 1) the result is noise), which is why the default mode is
// the tabulated evaluation above.  Every multiply and add is rounded on its own
// (__dmul_rn / __dadd_rn: no fused multiply-adds) so that this copy and the
// oracle's restatement of fmt.f90 round alike.
__device__ __forceinline__ double qk_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double qk_add(double a, double b) { return __dadd_rn(a, b); }
template <int N>
__device__ __forceinline__ double qk_horner(const double (&c)[N], double x) {
    double p = c[0];
#pragma unroll
    for (int i = 1; i < N; ++i) p = qk_add(qk_mul(p, x), c[i]);
    return p;
}

struct QuickFmtTop {
    double ww1, E, XINV;
    bool up;   // upward recursion from F_0 (else downward from F_M)
};

__device__ __forceinline__ QuickFmtTop quick_fmt_top(int M, double X) {
    constexpr double c33[3] = {1.9623264149430e-01, -4.9695241464490e-01, -6.0156581186481e-05};
    constexpr double c15[4] = {-1.8784686463512e-01, 2.2991849164985e-01, -4.9893752514047e-01,
                               -2.1916512131607e-05};
    constexpr double c10[7] = {4.6897511375022e-01, -6.9955602298985e-01, 5.3689283271887e-01,
                               -3.2883030418398e-01, 2.4645596956002e-01, -4.9984072848436e-01,
                               -3.1501078774085e-06};
    constexpr double c4[12] = {-2.62453564772299e-11, 3.24031041623823e-10, -3.614965656163e-09,
                               3.760256799971e-08, -3.553558319675e-07, 3.022556449731e-06,
                               -2.290098979647e-05, 1.526537461148e-04, -8.81947375894379e-04,
                               4.33207949514611e-03, -1.75257821619926e-02, 5.28406320615584e-02};
    constexpr double c2[12] = {-1.61702782425558e-10, 1.96215250865776e-09, -2.14234468198419e-08,
                               2.17216556336318e-07, -1.98850171329371e-06, 1.62429321438911e-05,
                               -1.16740298039895e-04, 7.24888732052332e-04, -3.79490003707156e-03,
                               1.61723488664661e-02, -5.29428148329736e-02, 1.15702180856167e-01};
    constexpr double c0[10] = {-8.36313918003957e-08, 1.21222603512827e-06, -1.15662609053481e-05,
                               9.25197374512647e-05, -6.40994113129432e-04, 3.78787044215009e-03,
                               -1.85185172458485e-02, 7.14285713298222e-02, -1.99999999997023e-01,
                               3.33333333333318e-01};
    constexpr double PIE4 = 3.14159265358979323846264338327950288 / 4.0;
    QuickFmtTop t;
    t.XINV = 1.0 / X;
    t.E = exp(-X);
    t.up = X > 1.0e-1 || (X > 1.0e-4 && M < 4);
    if (X > 5.0) {
        const double s = sqrt(qk_mul(PIE4, t.XINV));
        if (X > 33.0)
            t.ww1 = s;
        else if (X > 15.0)
            t.ww1 = qk_add(qk_mul(qk_horner(c33, t.XINV), t.E), s);
        else if (X > 10.0)
            t.ww1 = qk_add(qk_mul(qk_horner(c15, t.XINV), t.E), s);
        else
            t.ww1 = qk_add(qk_mul(qk_horner(c10, t.XINV), t.E), s);
    } else if (X > 1.0) {
        const double F1 = X > 3.0 ? qk_horner(c4, qk_add(X, -4.0)) : qk_horner(c2, qk_add(X, -2.0));
        t.ww1 = qk_add(qk_mul(qk_add(X, X), F1), t.E);
    } else if (t.up) {
        t.ww1 = qk_add(qk_mul(qk_add(X, X), qk_horner(c0, X)), t.E);
    } else {
        t.ww1 = qk_add(1.0, -X) / (double)(2 * M + 1);
    }
    return t;
}

// F_0..F_M at X by QUICK's formulas evaluated for the order MQ >= M (QUICK's CPU
// get2e evaluates at the shell quartet's order, which exceeds the class's M when
// SP shells take part; the branch, and in the downward case the starting value,
// depend on it), each multiplied by `scale`.
template <int M>
__device__ __forceinline__ void boys_quick_scaled(double X, double scale, double* F, int MQ) {
    const QuickFmtTop t = quick_fmt_top(MQ, X);
    double G[M + 1];
    if (t.up) {
        G[0] = t.ww1;
#pragma unroll
        for (int m = 1; m <= M; ++m)
            G[m] = qk_mul(qk_mul(qk_add(qk_mul((double)(2 * m - 1), G[m - 1]), -t.E), 0.5), t.XINV);
    } else {
        const double twot = qk_mul(X, 2.0);
        double f = t.ww1;
        for (int m = MQ - 1; m >= M; --m) f = qk_add(qk_mul(twot, f), t.E) / (double)(m * 2 + 1);
        G[M] = f;
#pragma unroll
        for (int m = M - 1; m >= 0; --m) G[m] = qk_add(qk_mul(twot, G[m + 1]), t.E) / (double)(m * 2 + 1);
    }
#pragma unroll
    for (int m = 0; m <= M; ++m) F[m] = G[m] * scale;
}

// F_m at X by QUICK's formulas for a total order M (the recursion runs from F_0
// up, or from F_M down, to m): one element, for the lane-parallel evaluation.
__device__ __forceinline__ double boys_quick_one(int m, int M, double X) {
    const QuickFmtTop t = quick_fmt_top(M, X);
    double f = t.ww1;
    if (t.up) {
        for (int j = 1; j <= m; ++j) f = qk_mul(qk_mul(qk_add(qk_mul((double)(2 * j - 1), f), -t.E), 0.5), t.XINV);
    } else {
        const double twot = qk_mul(X, 2.0);
        for (int j = M - 1; j >= m; --j) f = qk_add(qk_mul(twot, f), t.E) / (double)(j * 2 + 1);
    }
    return f;
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
