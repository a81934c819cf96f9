// CPU ORACLE -- test infrastructure only.
//
// A C++ restatement of QUICK's CPU closed-shell two-electron Fock build
// ("get2e") and of the per-geometry set-up it depends on.  It exists to check
// the CUDA path: only tests/, __graft_entry__.smoke() and bench.py's
// cpu_baseline / reference arm may load it.  Nothing in the quick_b200
// package links or calls it.
//
// Reference functions restated (paths relative to the QUICK source tree):
//   get_eri_precomputables  src/modules/include/eri.fh:62-154
//   schwarzoff/shellcutoff  src/modules/quick_cutoff_module.f90:54-253
//   classcutoff/classprim   src/modules/quick_cutoff_module.f90:255-588
//   cshell_density_cutoff   src/modules/include/cutoff.fh:16-92
//   get_cshell_eri          src/modules/include/eri.fh:161-203
//   cshell                  src/modules/include/eri.fh:209-442
//   iclass_cshell           src/modules/include/eri.fh:448-1058 (closed shell)
//   hrrwhole/lefthrr        src/subs/hrr.f90:7-857 (written generically here)
//   vertical + PSSS..       src/subs/hrr.f90:1051-3456, src/subs/spdfgh.f90
//                           (HGP eq. 6 written as one generic recursion)
//   copySym                 src/subs/copySym.f90:16-27
// Boys function: by default F_m(T) is evaluated accurately, with a Taylor
// expansion on a tabulated grid (table filled from the convergent series).
// src/subs/fmt.f90's fitted polynomials agree with it to ~1e-12 except in its
// small-X branch, F_M = (1 - X)/(2M + 1) for X <= 0.1 (M >= 4) or X <= 1e-4,
// which is first order in X; orc_set_boys_mode(1) switches to a restatement of
// fmt.f90 (boys_quick) to reproduce the reference's own numbers.
//
// One-electron integrals (overlap, kinetic, nuclear attraction) follow the
// Obara-Saika recursions over the normalize_basis representation
// (src/modules/quick_overlap_module.f90, quick_oei_module.f90); they are used
// only to run full SCF checks against the reference's saved energies.
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr double PI = 3.14159265358979323846264338327950288;
constexpr int MAXPRIM = 20;       // f-enabled reference build
constexpr int LMAX_SIDE = 6;      // f+f on one side
constexpr int NCART_TOT = 84;     // Cartesians with l+m+n <= 6
constexpr int MMAX = 12;          // 4*f

// ------------------------------------------------------------------ Cartesians
int g_cart_index[LMAX_SIDE + 3][LMAX_SIDE + 3][LMAX_SIDE + 3];
int g_cart_lmn[NCART_TOT][3];
int g_cart_start[LMAX_SIDE + 2];   // first index of total angular momentum L

void init_cart() {
    int idx = 0;
    for (int L = 0; L <= LMAX_SIDE; ++L) {
        g_cart_start[L] = idx;
        for (int l = L; l >= 0; --l)
            for (int m = L - l; m >= 0; --m) {
                int n = L - l - m;
                g_cart_index[l][m][n] = idx;
                g_cart_lmn[idx][0] = l; g_cart_lmn[idx][1] = m; g_cart_lmn[idx][2] = n;
                ++idx;
            }
    }
    g_cart_start[LMAX_SIDE + 1] = idx;
}
inline int ncart_upto(int L) { return g_cart_start[L + 1]; }

// ------------------------------------------------------------------ Boys
constexpr double BOYS_DT = 0.05;
constexpr int BOYS_NT = 721;          // T in [0, 36]
constexpr int BOYS_NM = MMAX + 1 + 8; // m up to MMAX + 8 Taylor terms
double g_boys_tab[BOYS_NT][BOYS_NM];

long double boys_series(int m, long double T) {
    // F_m(T) = exp(-T) sum_k (2T)^k / ((2m+1)(2m+3)...(2m+2k+1))
    long double term = 1.0L / (2 * m + 1), sum = term;
    for (int k = 1; k < 2000; ++k) {
        term *= 2.0L * T / (2 * m + 2 * k + 1);
        sum += term;
        if (term < sum * 1e-21L) break;
    }
    return std::exp(-T) * sum;
}

void init_boys() {
    for (int i = 0; i < BOYS_NT; ++i)
        for (int m = 0; m < BOYS_NM; ++m)
            g_boys_tab[i][m] = (double)boys_series(m, (long double)(i * BOYS_DT));
}

// F_0..F_M at T as QUICK computes it (src/subs/fmt.f90:13-85; the device copy,
// src/gpu/gpu_fmt.h:5-72, has the same branches): fitted polynomials in 1/X
// above X = 5, polynomials around X = 2 and 4 on (1, 5], a series-derived
// polynomial on (0.1, 1] (down to 1e-4 when M < 4), and below that
// F_M = (1 - X)/(2M + 1), followed by upward or downward recursion.  The last
// branch is first order in X (relative error up to ~2% in F_M at X = 0.1, M = 4),
// so the reference's integrals differ from exact ones there.
// One multiply or add, rounded on its own (the empty asm keeps the compiler from
// fusing it with a neighbour into an FMA): boys_quick rounds exactly as the
// device copy of it does, which uses __dmul_rn / __dadd_rn.
inline double mul_rn(double a, double b) {
    double r = a * b;
    asm volatile("" : "+x"(r));
    return r;
}
inline double add_rn(double a, double b) {
    double r = a + b;
    asm volatile("" : "+x"(r));
    return r;
}
// Horner's rule, c[0] the leading coefficient, one rounding per operation
inline double horner_rn(const double* c, int n, double x) {
    double p = c[0];
    for (int i = 1; i < n; ++i) p = add_rn(mul_rn(p, x), c[i]);
    return p;
}

// Sensitivity probe: exp(-X) one ulp up inside boys_quick (0 = off).  QUICK's
// recursion is unstable in parts of its range, so its results depend on the last
// bit of the exp it links; this shows by how much.
int g_exp_ulp = 0;

void boys_quick(int M, double X, double* F) {
    static const double c33[] = {1.9623264149430e-01, -4.9695241464490e-01, -6.0156581186481e-05};
    static const double c15[] = {-1.8784686463512e-01, 2.2991849164985e-01, -4.9893752514047e-01,
                                 -2.1916512131607e-05};
    static const double c10[] = {4.6897511375022e-01, -6.9955602298985e-01, 5.3689283271887e-01,
                                 -3.2883030418398e-01, 2.4645596956002e-01, -4.9984072848436e-01,
                                 -3.1501078774085e-06};
    static const double c4[] = {-2.62453564772299e-11, 3.24031041623823e-10, -3.614965656163e-09,
                                3.760256799971e-08, -3.553558319675e-07, 3.022556449731e-06,
                                -2.290098979647e-05, 1.526537461148e-04, -8.81947375894379e-04,
                                4.33207949514611e-03, -1.75257821619926e-02, 5.28406320615584e-02};
    static const double c2[] = {-1.61702782425558e-10, 1.96215250865776e-09, -2.14234468198419e-08,
                                2.17216556336318e-07, -1.98850171329371e-06, 1.62429321438911e-05,
                                -1.16740298039895e-04, 7.24888732052332e-04, -3.79490003707156e-03,
                                1.61723488664661e-02, -5.29428148329736e-02, 1.15702180856167e-01};
    static const double c0[] = {-8.36313918003957e-08, 1.21222603512827e-06, -1.15662609053481e-05,
                                9.25197374512647e-05, -6.40994113129432e-04, 3.78787044215009e-03,
                                -1.85185172458485e-02, 7.14285713298222e-02, -1.99999999997023e-01,
                                3.33333333333318e-01};
    const double PIE4 = PI / 4.0;
    const double XINV = 1.0 / X;
    const double E = g_exp_ulp ? std::nextafter(std::exp(-X), 2.0) : std::exp(-X);
    double WW1;
    if (X > 5.0) {
        const double s = std::sqrt(mul_rn(PIE4, XINV));
        if (X > 33.0)
            WW1 = s;
        else if (X > 15.0)
            WW1 = add_rn(mul_rn(horner_rn(c33, 3, XINV), E), s);
        else if (X > 10.0)
            WW1 = add_rn(mul_rn(horner_rn(c15, 4, XINV), E), s);
        else
            WW1 = add_rn(mul_rn(horner_rn(c10, 7, XINV), E), s);
    } else if (X > 1.0) {
        const double F1 = X > 3.0 ? horner_rn(c4, 12, add_rn(X, -4.0)) : horner_rn(c2, 12, add_rn(X, -2.0));
        WW1 = add_rn(mul_rn(add_rn(X, X), F1), E);
    } else if (X > 1.0e-1 || (X > 1.0e-4 && M < 4)) {
        WW1 = add_rn(mul_rn(add_rn(X, X), horner_rn(c0, 10, X)), E);
    } else {
        WW1 = add_rn(1.0, -X) / (double)(2 * M + 1);
    }
    if (X > 1.0e-1 || (X > 1.0e-4 && M < 4)) {
        F[0] = WW1;
        for (int m = 1; m <= M; ++m)
            F[m] = mul_rn(mul_rn(add_rn(mul_rn((double)(2 * m - 1), F[m - 1]), -E), 0.5), XINV);
    } else {
        F[M] = WW1;
        const double twot = mul_rn(X, 2.0);
        for (int m = M - 1; m >= 0; --m) F[m] = add_rn(mul_rn(twot, F[m + 1]), E) / (double)(m * 2 + 1);
    }
}

// Boys function used by the integral code: 0 = accurate (the tabulated Taylor
// form below), 1 = QUICK's own (boys_quick), to compare with the reference's
// implementations at the last digits.
int g_boys_mode = 0;

// F_0..F_M at T
void boys(int M, double T, double* F) {
    if (g_boys_mode == 1) { boys_quick(M, T, F); return; }
    if (T < 36.0) {
        int k = (int)(T / BOYS_DT + 0.5);
        double d = T - k * BOYS_DT;
        const double* t = g_boys_tab[k];
        double fm = 0.0, c = 1.0;
        for (int j = 0; j < 8; ++j) { fm += t[M + j] * c; c *= -d / (j + 1); }
        F[M] = fm;
        double e = std::exp(-T);
        for (int m = M; m > 0; --m) F[m - 1] = (2.0 * T * F[m] + e) / (2 * m - 1);
    } else {
        double e = std::exp(-T);
        F[0] = 0.5 * std::sqrt(PI / T);
        for (int m = 0; m < M; ++m) F[m + 1] = ((2 * m + 1) * F[m] - e) / (2.0 * T);
    }
}

// ------------------------------------------------------------------ basis view
struct Basis {
    int natom, nshell, nbasis, jbasis;
    std::vector<double> xyz;                 // 3*natom
    std::vector<int> kstart, katom, ktype, kprim, ksumtype, qstart, qfinal;
    std::vector<int> qsbasis, qfbasis;       // nshell*4 (col-major (nshell,4))
    std::vector<double> gccoeff, gcexpo;     // MAXPRIM*nbasis
    std::vector<double> cons;                // nbasis
    std::vector<int> klmn;                   // 3*nbasis
    // precomputables
    std::vector<double> Apri, Kpri, Ppri;    // jbasis^2, jbasis^2, 3*jbasis^2
    std::vector<double> Xcoeff;              // jbasis^2*16: [(a*jbasis+b)*16 + I*4+J]
    double A(int s, int k) const { return xyz[3 * (katom[s] - 1) + k]; }
    int qs(int s, int L) const { return qsbasis[s + nshell * L]; }
    int qf(int s, int L) const { return qfbasis[s + nshell * L]; }
    double X(int a, int b, int I, int J) const { return Xcoeff[((size_t)a * jbasis + b) * 16 + I * 4 + J]; }
};

void precompute(Basis& B) {
    // src/modules/include/eri.fh:62-154
    int jb = B.jbasis;
    B.Apri.assign((size_t)jb * jb, 0.0);
    B.Kpri.assign((size_t)jb * jb, 0.0);
    B.Ppri.assign((size_t)3 * jb * jb, 0.0);
    B.Xcoeff.assign((size_t)jb * jb * 16, 0.0);
    for (int ics = 0; ics < B.nshell; ++ics)
        for (int ips = 0; ips < B.kprim[ics]; ++ips)
            for (int jcs = 0; jcs < B.nshell; ++jcs)
                for (int jps = 0; jps < B.kprim[jcs]; ++jps) {
                    int NA = B.kstart[ics] - 1 + ips, NB = B.kstart[jcs] - 1 + jps;
                    int fi = B.ksumtype[ics] - 1, fj = B.ksumtype[jcs] - 1;
                    double AA = B.gcexpo[ips + MAXPRIM * fi];
                    double BB = B.gcexpo[jps + MAXPRIM * fj];
                    size_t ab = (size_t)NA * jb + NB;
                    B.Apri[ab] = AA + BB;
                    double d2 = 0.0;
                    for (int k = 0; k < 3; ++k) {
                        double xa = B.A(ics, k), xb = B.A(jcs, k);
                        d2 += (xa - xb) * (xa - xb);
                        B.Ppri[3 * ab + k] = (xa * AA + xb * BB) / (AA + BB);
                    }
                    double DAB = std::sqrt(d2);
                    B.Kpri[ab] = std::exp(-AA * BB / (AA + BB) * (DAB * DAB)) / (AA + BB);
                    for (int I = B.qstart[ics]; I <= B.qfinal[ics]; ++I)
                        for (int J = B.qstart[jcs]; J <= B.qfinal[jcs]; ++J)
                            B.Xcoeff[ab * 16 + I * 4 + J] = B.Kpri[ab]
                                * B.gccoeff[ips + MAXPRIM * (fi + I)]
                                * B.gccoeff[jps + MAXPRIM * (fj + J)];
                }
}

// ------------------------------------------------------------------ VRR
// Per-thread workspace.  V[m][e][f] = [e0|f0]^(m) for Cartesian indices e, f.
struct Work {
    std::vector<double> V;      // (MMAX+1) * 84 * 84
    std::vector<double> Y;      // ITT * 84 * 84 stored primitive results (compact)
    std::vector<double> X44;
    std::vector<double> store;  // 84*84
    Work() : V((size_t)(MMAX + 1) * NCART_TOT * NCART_TOT), store(NCART_TOT * NCART_TOT) {}
    double& v(int m, int e, int f) { return V[((size_t)m * NCART_TOT + e) * NCART_TOT + f]; }
};

struct PrimGeom {
    double PA[3], QC[3], WP[3], WQ[3];
    double oo2z, oo2e, oo2ze, rho_z, rho_e;  // 1/2zeta, 1/2eta, 1/2(zeta+eta), eta/(z+e), zeta/(z+e)
};

// Fill [e0|f0]^(m) for e < ncart_upto(Lab), f < ncart_upto(Lcd), starting from
// V[m][0][0] already set.  HGP eq. 6 and its ket analogue; the recursion
// direction is the first Cartesian axis with a non-zero exponent.
void vrr(Work& W, const PrimGeom& G, int Lab, int Lcd) {
    int Mtot = Lab + Lcd;
    // bra build, f = 0
    for (int L = 1; L <= Lab; ++L)
        for (int e = g_cart_start[L]; e < g_cart_start[L + 1]; ++e) {
            const int* lmn = g_cart_lmn[e];
            int i = lmn[0] ? 0 : (lmn[1] ? 1 : 2);
            int a1[3] = {lmn[0], lmn[1], lmn[2]};
            a1[i] -= 1;
            int e1 = g_cart_index[a1[0]][a1[1]][a1[2]];
            int e2 = -1;
            double n2 = a1[i];
            if (a1[i] > 0) { int a2[3] = {a1[0], a1[1], a1[2]}; a2[i] -= 1; e2 = g_cart_index[a2[0]][a2[1]][a2[2]]; }
            for (int m = 0; m <= Mtot - L; ++m) {
                double val = G.PA[i] * W.v(m, e1, 0) + G.WP[i] * W.v(m + 1, e1, 0);
                if (e2 >= 0) val += n2 * G.oo2z * (W.v(m, e2, 0) - G.rho_z * W.v(m + 1, e2, 0));
                W.v(m, e, 0) = val;
            }
        }
    // ket build
    for (int L = 1; L <= Lcd; ++L)
        for (int f = g_cart_start[L]; f < g_cart_start[L + 1]; ++f) {
            const int* lmn = g_cart_lmn[f];
            int i = lmn[0] ? 0 : (lmn[1] ? 1 : 2);
            int c1[3] = {lmn[0], lmn[1], lmn[2]};
            c1[i] -= 1;
            int f1 = g_cart_index[c1[0]][c1[1]][c1[2]];
            int f2 = -1;
            double n2 = c1[i];
            if (c1[i] > 0) { int c2[3] = {c1[0], c1[1], c1[2]}; c2[i] -= 1; f2 = g_cart_index[c2[0]][c2[1]][c2[2]]; }
            for (int Le = 0; Le <= Lab; ++Le)
                for (int e = g_cart_start[Le]; e < g_cart_start[Le + 1]; ++e) {
                    const int* alm = g_cart_lmn[e];
                    int em = -1;
                    double na = alm[i];
                    if (alm[i] > 0) { int a1[3] = {alm[0], alm[1], alm[2]}; a1[i] -= 1; em = g_cart_index[a1[0]][a1[1]][a1[2]]; }
                    for (int m = 0; m <= Mtot - L - Le; ++m) {
                        double val = G.QC[i] * W.v(m, e, f1) + G.WQ[i] * W.v(m + 1, e, f1);
                        if (f2 >= 0) val += n2 * G.oo2e * (W.v(m, e, f2) - G.rho_e * W.v(m + 1, e, f2));
                        if (em >= 0) val += na * G.oo2ze * W.v(m + 1, em, f1);
                        W.v(m, e, f) = val;
                    }
                }
        }
}

// ------------------------------------------------------------------ HRR
// (a b| = sum_e coef * [e 0|  with (a, b+1_i| = (a+1_i, b| + (A-B)_i (a, b|
// (same relation as lefthrr, src/subs/hrr.f90:289-857).
void hrr_expand(const int a[3], const int b[3], const double AB[3], double coef,
                std::vector<std::pair<int, double>>& out) {
    if (b[0] + b[1] + b[2] == 0) {
        out.emplace_back(g_cart_index[a[0]][a[1]][a[2]], coef);
        return;
    }
    int i = b[0] ? 0 : (b[1] ? 1 : 2);
    int b1[3] = {b[0], b[1], b[2]};
    b1[i] -= 1;
    int ap[3] = {a[0], a[1], a[2]};
    ap[i] += 1;
    hrr_expand(ap, b1, AB, coef, out);
    if (AB[i] != 0.0) hrr_expand(a, b1, AB, coef * AB[i], out);
}

// ------------------------------------------------------------------ one quartet
// cshell + iclass_cshell for shells II,JJ,KK,LL (0-based); digestion into G
// (nbasis x nbasis column-major, element (row r, col c) at r + n*c), following
// the index-equality branches of src/modules/include/eri.fh:649-1050.
struct Ctx {
    const Basis* B;
    const double* dense;      // nbasis^2 col-major: the density of the J terms
    const double* cutmatrix;  // nshell^2
    const double* cutprim;    // jbasis^2
    double integralCutoff, primLimit;
    // QUICK's GPU path screens two more things than the CPU get2e: only shell
    // pairs with Y > 1e-10 enter its pair list (src/gpu/cuda/gpu.cu:929-1030) and
    // integrals with |Y| <= integralCutoff are not digested
    // (src/gpu/gpu_get2e_subs.h:389).  gpu_screens reproduces both, to compare
    // with that implementation; off, this is the CPU get2e.
    bool gpu_screens = false;
    // density of the K terms when it differs from `dense` (an open-shell matrix: 2 Da
    // or 2 Db against J's Da + Db); null = the same
    const double* dense_k = nullptr;
};

inline double& O(double* G, int n, int r, int c) { return G[(size_t)(r - 1) + (size_t)n * (c - 1)]; }
inline double Dn(const double* D, int n, int r, int c) { return D[(size_t)(r - 1) + (size_t)n * (c - 1)]; }

void cshell_quartet(const Ctx& C, Work& W, int II, int JJ, int KK, int LL, double dnmax, double* Gm) {
    const Basis& B = *C.B;
    const int jb = B.jbasis, n = B.nbasis;
    double RA[3], RB[3], RC[3], RD[3];
    for (int k = 0; k < 3; ++k) { RA[k] = B.A(II, k); RB[k] = B.A(JJ, k); RC[k] = B.A(KK, k); RD[k] = B.A(LL, k); }
    int NII1 = B.qstart[II], NII2 = B.qfinal[II], NJJ1 = B.qstart[JJ], NJJ2 = B.qfinal[JJ];
    int NKK1 = B.qstart[KK], NKK2 = B.qfinal[KK], NLL1 = B.qstart[LL], NLL2 = B.qfinal[LL];
    int Lab = NII2 + NJJ2, Lcd = NKK2 + NLL2, Mtot = Lab + Lcd;
    int ne = ncart_upto(Lab), nf = ncart_upto(Lcd);
    const int e0 = g_cart_start[NII1], f0 = g_cart_start[NKK1];
    const int nstore_e = ne - e0, nstore_f = nf - f0;

    // primitive loop (eri.fh:260-418): store surviving [e0|f0]^(0) in order ITT
    W.Y.clear();
    double FM[MMAX + 2];
    for (int jjj = 0; jjj < B.kprim[JJ]; ++jjj) {
        int Nj = B.kstart[JJ] - 1 + jjj;
        for (int iii = 0; iii < B.kprim[II]; ++iii) {
            int Ni = B.kstart[II] - 1 + iii;
            size_t ij = (size_t)Ni * jb + Nj;
            double AB = B.Apri[ij];
            double cut1 = dnmax * C.cutprim[ij];
            const double* P = &B.Ppri[3 * ij];
            for (int lll = 0; lll < B.kprim[LL]; ++lll) {
                int Nl = B.kstart[LL] - 1 + lll;
                for (int kkk = 0; kkk < B.kprim[KK]; ++kkk) {
                    int Nk = B.kstart[KK] - 1 + kkk;
                    size_t kl = (size_t)Nk * jb + Nl;
                    if (!(cut1 * C.cutprim[kl] > C.primLimit)) continue;
                    double CD = B.Apri[kl];
                    double ABCD = AB + CD;
                    double ROU = AB * CD / ABCD;
                    const double* Q = &B.Ppri[3 * kl];
                    PrimGeom Gg;
                    double RPQ = 0.0;
                    for (int k = 0; k < 3; ++k) {
                        double Wk = (P[k] * AB + Q[k] * CD) / ABCD;
                        double d = P[k] - Q[k];
                        RPQ += d * d;
                        Gg.PA[k] = P[k] - RA[k];
                        Gg.QC[k] = Q[k] - RC[k];
                        Gg.WP[k] = Wk - P[k];
                        Gg.WQ[k] = Wk - Q[k];
                    }
                    Gg.oo2z = 0.5 / AB; Gg.oo2e = 0.5 / CD; Gg.oo2ze = 0.5 / ABCD;
                    Gg.rho_z = CD / ABCD; Gg.rho_e = AB / ABCD;
                    double T = RPQ * ROU;
                    boys(Mtot, T, FM);
                    double s = 1.0 / std::sqrt(ABCD);
                    for (int m = 0; m <= Mtot; ++m) W.v(m, 0, 0) = FM[m] * s;
                    vrr(W, Gg, Lab, Lcd);
                    for (int e = e0; e < ne; ++e)
                        for (int f = f0; f < nf; ++f) W.Y.push_back(W.v(0, e, f));
                }
            }
        }
    }
    const size_t stride = (size_t)nstore_e * nstore_f;
    const int ITT = (int)(W.Y.size() / (stride ? stride : 1));

    const double X0 = 2.0 * std::pow(PI, 2.5);
    std::vector<std::pair<int, double>> hl, hr;
    double ABv[3] = {RA[0] - RB[0], RA[1] - RB[1], RA[2] - RB[2]};
    double CDv[3] = {RC[0] - RD[0], RC[1] - RD[1], RC[2] - RD[2]};

    for (int I = NII1; I <= NII2; ++I)
        for (int J = NJJ1; J <= NJJ2; ++J)
            for (int K = NKK1; K <= NKK2; ++K)
                for (int L = NLL1; L <= NLL2; ++L) {
                    // contraction (eri.fh:480-545)
                    W.X44.clear();
                    for (int jjj = 0; jjj < B.kprim[JJ]; ++jjj) {
                        int Nj = B.kstart[JJ] - 1 + jjj;
                        for (int iii = 0; iii < B.kprim[II]; ++iii) {
                            int Ni = B.kstart[II] - 1 + iii;
                            double X2 = X0 * B.X(Ni, Nj, I, J);
                            double cut1 = dnmax * C.cutprim[(size_t)Ni * jb + Nj];
                            for (int lll = 0; lll < B.kprim[LL]; ++lll) {
                                int Nl = B.kstart[LL] - 1 + lll;
                                for (int kkk = 0; kkk < B.kprim[KK]; ++kkk) {
                                    int Nk = B.kstart[KK] - 1 + kkk;
                                    if (cut1 * C.cutprim[(size_t)Nk * jb + Nl] > C.primLimit)
                                        W.X44.push_back(X2 * B.X(Nk, Nl, K, L));
                                }
                            }
                        }
                    }
                    int eA = g_cart_start[I], eB = ncart_upto(I + J);
                    int fC = g_cart_start[K], fD = ncart_upto(K + L);
                    for (int e = eA; e < eB; ++e)
                        for (int f = fC; f < fD; ++f) {
                            double y = 0.0;
                            size_t off = (size_t)(e - e0) * nstore_f + (f - f0);
                            for (int t = 0; t < ITT; ++t) y += W.X44[t] * W.Y[t * stride + off];
                            W.store[e * NCART_TOT + f] = y;
                        }

                    int III1 = B.ksumtype[II] + B.qs(II, I), III2 = B.ksumtype[II] + B.qf(II, I);
                    int JJJ1 = B.ksumtype[JJ] + B.qs(JJ, J), JJJ2 = B.ksumtype[JJ] + B.qf(JJ, J);
                    int KKK1 = B.ksumtype[KK] + B.qs(KK, K), KKK2 = B.ksumtype[KK] + B.qf(KK, K);
                    int LLL1 = B.ksumtype[LL] + B.qs(LL, L), LLL2 = B.ksumtype[LL] + B.qf(LL, L);

                    auto hrrwhole = [&](int iii, int jjj, int kkk, int lll) -> double {
                        const int* a = &B.klmn[3 * (iii - 1)];
                        const int* b = &B.klmn[3 * (jjj - 1)];
                        const int* c = &B.klmn[3 * (kkk - 1)];
                        const int* d = &B.klmn[3 * (lll - 1)];
                        hl.clear(); hr.clear();
                        hrr_expand(a, b, ABv, 1.0, hl);
                        hrr_expand(c, d, CDv, 1.0, hr);
                        double y = 0.0;
                        for (auto& l : hl)
                            for (auto& r : hr) y += l.second * r.second * W.store[l.first * NCART_TOT + r.first];
                        return y * B.cons[iii - 1] * B.cons[jjj - 1] * B.cons[kkk - 1] * B.cons[lll - 1];
                    };
                    // J terms read DJ, K terms read DK: the closed-shell build has DJ = DK = D;
                    // the open-shell (OSHELL) branches of eri.fh are the same updates with
                    // DJ = Da + Db and, for the alpha (beta) matrix, DK = 2 Da (2 Db), the
                    // K coefficients of the closed shell halved against the total density.
                    const double* DJ = C.dense;
                    const double* DK = C.dense_k ? C.dense_k : C.dense;
                    const double hx = 1.0;  // x_hybrid_coeff for HF
                    auto J = [&](int r, int cc) { return Dn(DJ, n, r, cc); };
                    auto K = [&](int r, int cc) { return Dn(DK, n, r, cc); };
                    if (II < JJ && II < KK && KK < LL) {
                        for (int III = III1; III <= III2; ++III)
                            for (int JJJ = JJJ1; JJJ <= JJJ2; ++JJJ)
                                for (int KKK = KKK1; KKK <= KKK2; ++KKK)
                                    for (int LLL = LLL1; LLL <= LLL2; ++LLL) {
                                        double Y = hrrwhole(III, JJJ, KKK, LLL);
                                        if (C.gpu_screens && !(std::fabs(Y) > C.integralCutoff)) continue;
                                        O(Gm, n, JJJ, III) += 2.0 * J(LLL, KKK) * Y;
                                        O(Gm, n, LLL, KKK) += 2.0 * J(JJJ, III) * Y;
                                        O(Gm, n, KKK, III) -= hx * 0.5 * K(LLL, JJJ) * Y;
                                        O(Gm, n, LLL, III) -= hx * 0.5 * K(KKK, JJJ) * Y;
                                        O(Gm, n, JJJ, KKK) -= hx * 0.5 * K(LLL, III) * Y;
                                        O(Gm, n, JJJ, LLL) -= hx * 0.5 * K(KKK, III) * Y;
                                        O(Gm, n, KKK, JJJ) -= hx * 0.5 * K(LLL, III) * Y;
                                        O(Gm, n, LLL, JJJ) -= hx * 0.5 * K(KKK, III) * Y;
                                    }
                    } else {
                        for (int III = III1; III <= III2; ++III)
                            for (int JJJ = std::max(III, JJJ1); JJJ <= JJJ2; ++JJJ)
                                for (int KKK = std::max(III, KKK1); KKK <= KKK2; ++KKK)
                                    for (int LLL = std::max(KKK, LLL1); LLL <= LLL2; ++LLL) {
                                        if (III < KKK) {
                                            double Y = hrrwhole(III, JJJ, KKK, LLL);
                                            if (C.gpu_screens && !(std::fabs(Y) > C.integralCutoff)) continue;
                                            if (III < JJJ && KKK < LLL) {
                                                O(Gm, n, JJJ, III) += 2.0 * J(LLL, KKK) * Y;
                                                O(Gm, n, LLL, KKK) += 2.0 * J(JJJ, III) * Y;
                                                O(Gm, n, KKK, III) -= hx * 0.5 * K(LLL, JJJ) * Y;
                                                O(Gm, n, LLL, III) -= hx * 0.5 * K(KKK, JJJ) * Y;
                                                O(Gm, n, JJJ, KKK) -= hx * 0.5 * K(LLL, III) * Y;
                                                O(Gm, n, JJJ, LLL) -= hx * 0.5 * K(KKK, III) * Y;
                                                O(Gm, n, KKK, JJJ) -= hx * 0.5 * K(LLL, III) * Y;
                                                O(Gm, n, LLL, JJJ) -= hx * 0.5 * K(KKK, III) * Y;
                                            } else if (III == JJJ && KKK == LLL) {
                                                O(Gm, n, III, III) += J(KKK, KKK) * Y;
                                                O(Gm, n, KKK, KKK) += J(III, III) * Y;
                                                O(Gm, n, KKK, III) -= hx * 0.5 * K(KKK, III) * Y;
                                            } else if (JJJ == KKK && JJJ == LLL) {
                                                O(Gm, n, JJJ, III) += J(JJJ, JJJ) * Y - hx * 0.5 * K(JJJ, JJJ) * Y;
                                                O(Gm, n, JJJ, JJJ) += 2.0 * J(JJJ, III) * Y - hx * K(JJJ, III) * Y;
                                            } else if (KKK == LLL && III < JJJ && JJJ != KKK) {
                                                O(Gm, n, JJJ, III) += J(KKK, KKK) * Y;
                                                O(Gm, n, KKK, KKK) += 2.0 * J(JJJ, III) * Y;
                                                O(Gm, n, KKK, III) -= hx * 0.5 * K(KKK, JJJ) * Y;
                                                O(Gm, n, KKK, JJJ) -= hx * 0.5 * K(KKK, III) * Y;
                                                O(Gm, n, JJJ, KKK) -= hx * 0.5 * K(KKK, III) * Y;
                                            } else if (III == JJJ && KKK < LLL) {
                                                O(Gm, n, LLL, KKK) += J(III, III) * Y;
                                                O(Gm, n, III, III) += 2.0 * J(LLL, KKK) * Y;
                                                O(Gm, n, KKK, III) -= hx * 0.5 * K(LLL, III) * Y;
                                                O(Gm, n, LLL, III) -= hx * 0.5 * K(KKK, III) * Y;
                                            }
                                        } else if (JJJ <= LLL) {
                                            double Y = hrrwhole(III, JJJ, KKK, LLL);
                                            if (C.gpu_screens && !(std::fabs(Y) > C.integralCutoff)) continue;
                                            if (III == JJJ && III == KKK && III == LLL) {
                                                O(Gm, n, III, III) += J(III, III) * Y - hx * 0.5 * K(III, III) * Y;
                                            } else if (III == JJJ && III == KKK && III < LLL) {
                                                O(Gm, n, LLL, III) += J(III, III) * Y - hx * 0.5 * K(III, III) * Y;
                                                O(Gm, n, III, III) += 2.0 * J(LLL, III) * Y - hx * K(LLL, III) * Y;
                                            } else if (III == KKK && JJJ == LLL && III < JJJ) {
                                                O(Gm, n, JJJ, III) += 2.0 * J(JJJ, III) * Y - hx * 0.5 * K(JJJ, III) * Y;
                                                O(Gm, n, JJJ, JJJ) -= hx * 0.5 * K(III, III) * Y;
                                                O(Gm, n, III, III) -= hx * 0.5 * K(JJJ, JJJ) * Y;
                                            } else if (III == KKK && III < JJJ && JJJ < LLL) {
                                                O(Gm, n, JJJ, III) += 2.0 * J(LLL, III) * Y - hx * 0.5 * K(LLL, III) * Y;
                                                O(Gm, n, LLL, III) += 2.0 * J(JJJ, III) * Y - hx * 0.5 * K(JJJ, III) * Y;
                                                O(Gm, n, III, III) -= hx * 1.0 * K(LLL, JJJ) * Y;
                                                O(Gm, n, LLL, JJJ) -= hx * 0.5 * K(III, III) * Y;
                                            }
                                        }
                                    }
                    }
                }
}

double dnmax_of(const Ctx& C, int II, int JJ, int KK, int LL) {
    int ns = C.B->nshell;
    auto cm = [&](int a, int b) { return C.cutmatrix[a + (size_t)ns * b]; };
    return std::max({4.0 * cm(II, JJ), 4.0 * cm(KK, LL), cm(II, LL), cm(II, KK), cm(JJ, KK), cm(JJ, LL)});
}

// ------------------------------------------------------------------ Schwarz
// shellcutoff / classcutoff / classprim: Ycutoff(II,JJ) = sqrt(max |(ij|ij)|),
// cutprim(i,j) = sqrt(max |primitive (ij|ij)|) over the components.
void shell_cutoff(const Basis& B, Work& W, int II, int JJ, double* Ycut, double* cutprim) {
    const int jb = B.jbasis;
    int KK = II, LL = JJ;
    double RA[3], RB[3];
    for (int k = 0; k < 3; ++k) { RA[k] = B.A(II, k); RB[k] = B.A(JJ, k); }
    int NII1 = B.qstart[II], NII2 = B.qfinal[II], NJJ1 = B.qstart[JJ], NJJ2 = B.qfinal[JJ];
    int Lab = NII2 + NJJ2, Mtot = 2 * Lab;
    int ne = ncart_upto(Lab), e0 = g_cart_start[NII1];
    int nst = ne - e0;
    size_t stride = (size_t)nst * nst;
    int npi = B.kprim[II], npj = B.kprim[JJ];
    // all primitive quartets (no screening), and the diagonal ones per prim pair
    std::vector<double> Yall;
    std::vector<double> Ydiag((size_t)npi * npj * stride);
    double FM[MMAX + 2];
    double ABv[3] = {RA[0] - RB[0], RA[1] - RB[1], RA[2] - RB[2]};
    for (int jjj = 0; jjj < npj; ++jjj) {
        int Nj = B.kstart[JJ] - 1 + jjj;
        for (int iii = 0; iii < npi; ++iii) {
            int Ni = B.kstart[II] - 1 + iii;
            size_t ij = (size_t)Ni * jb + Nj;
            double AB = B.Apri[ij];
            const double* P = &B.Ppri[3 * ij];
            for (int lll = 0; lll < B.kprim[LL]; ++lll) {
                int Nl = B.kstart[LL] - 1 + lll;
                for (int kkk = 0; kkk < B.kprim[KK]; ++kkk) {
                    int Nk = B.kstart[KK] - 1 + kkk;
                    size_t kl = (size_t)Nk * jb + Nl;
                    double CD = B.Apri[kl], ABCD = AB + CD, ROU = AB * CD / ABCD;
                    const double* Q = &B.Ppri[3 * kl];
                    PrimGeom Gg;
                    double RPQ = 0.0;
                    for (int k = 0; k < 3; ++k) {
                        double Wk = (P[k] * AB + Q[k] * CD) / ABCD;
                        double d = P[k] - Q[k];
                        RPQ += d * d;
                        Gg.PA[k] = P[k] - RA[k];
                        Gg.QC[k] = Q[k] - RA[k];   // RC = RA for the diagonal quartet
                        Gg.WP[k] = Wk - P[k];
                        Gg.WQ[k] = Wk - Q[k];
                    }
                    Gg.oo2z = 0.5 / AB; Gg.oo2e = 0.5 / CD; Gg.oo2ze = 0.5 / ABCD;
                    Gg.rho_z = CD / ABCD; Gg.rho_e = AB / ABCD;
                    boys(Mtot, RPQ * ROU, FM);
                    double s = 1.0 / std::sqrt(ABCD);
                    for (int m = 0; m <= Mtot; ++m) W.v(m, 0, 0) = FM[m] * s;
                    vrr(W, Gg, Lab, Lab);
                    for (int e = e0; e < ne; ++e)
                        for (int f = e0; f < ne; ++f) {
                            double v = W.v(0, e, f);
                            Yall.push_back(v);
                            if (kkk == iii && lll == jjj)
                                Ydiag[((size_t)(iii * npj + jjj)) * stride + (size_t)(e - e0) * nst + (f - e0)] = v;
                        }
                }
            }
        }
    }
    const double X0 = 2.0 * std::pow(PI, 2.5);
    std::vector<std::pair<int, double>> hl;
    auto diag_value = [&](const std::vector<double>& store_in, int I, int J) {
        // max over III in I-part, JJJ in J-part of |(III JJJ|III JJJ)| * cons^4
        double ymax = 0.0;
        int III1 = B.ksumtype[II] + B.qs(II, I), III2 = B.ksumtype[II] + B.qf(II, I);
        int JJJ1 = B.ksumtype[JJ] + B.qs(JJ, J), JJJ2 = B.ksumtype[JJ] + B.qf(JJ, J);
        for (int III = III1; III <= III2; ++III)
            for (int JJJ = JJJ1; JJJ <= JJJ2; ++JJJ) {
                hl.clear();
                hrr_expand(&B.klmn[3 * (III - 1)], &B.klmn[3 * (JJJ - 1)], ABv, 1.0, hl);
                double y = 0.0;
                for (auto& l : hl)
                    for (auto& r : hl) y += l.second * r.second * store_in[(size_t)(l.first - e0) * nst + (r.first - e0)];
                double c = B.cons[III - 1] * B.cons[JJJ - 1];
                y *= c * c;
                ymax = std::max(ymax, std::fabs(y));
            }
        return ymax;
    };
    // cutprim per primitive pair (classprim)
    std::vector<double> st(stride);
    for (int iii = 0; iii < npi; ++iii)
        for (int jjj = 0; jjj < npj; ++jjj) {
            int Ni = B.kstart[II] - 1 + iii, Nj = B.kstart[JJ] - 1 + jjj;
            double ymax = 0.0;
            for (int I = NII1; I <= NII2; ++I)
                for (int J = NJJ1; J <= NJJ2; ++J) {
                    double x = X0 * B.X(Ni, Nj, I, J);
                    const double* yd = &Ydiag[((size_t)(iii * npj + jjj)) * stride];
                    for (size_t t = 0; t < stride; ++t) st[t] = yd[t] * x * x;
                    ymax = std::max(ymax, diag_value(st, I, J));
                }
            double v = std::sqrt(ymax);
            cutprim[(size_t)Ni * jb + Nj] = v;
            cutprim[(size_t)Nj * jb + Ni] = v;
        }
    // Ycutoff (classcutoff): contracted diagonal quartet
    double ymax = 0.0;
    for (int I = NII1; I <= NII2; ++I)
        for (int J = NJJ1; J <= NJJ2; ++J) {
            std::fill(st.begin(), st.end(), 0.0);
            size_t itt = 0;
            for (int jjj = 0; jjj < npj; ++jjj) {
                int Nj = B.kstart[JJ] - 1 + jjj;
                for (int iii = 0; iii < npi; ++iii) {
                    int Ni = B.kstart[II] - 1 + iii;
                    double X2 = X0 * B.X(Ni, Nj, I, J);
                    for (int lll = 0; lll < npj; ++lll) {
                        int Nl = B.kstart[LL] - 1 + lll;
                        for (int kkk = 0; kkk < npi; ++kkk) {
                            int Nk = B.kstart[KK] - 1 + kkk;
                            double x44 = X2 * B.X(Nk, Nl, I, J);
                            const double* y = &Yall[itt * stride];
                            for (size_t t = 0; t < stride; ++t) st[t] += x44 * y[t];
                            ++itt;
                        }
                    }
                }
            }
            ymax = std::max(ymax, diag_value(st, I, J));
        }
    double v = std::sqrt(ymax);
    Ycut[II + (size_t)B.nshell * JJ] = v;
    Ycut[JJ + (size_t)B.nshell * II] = v;
}

// ------------------------------------------------------------------ 1e ints
// Obara-Saika overlap/kinetic and nuclear attraction over primitive pairs.
struct OEIBasis {
    int nbasis, maxcontract, natom;
    const int* ncontract; const int* itype; const double* aexp; const double* dcoeff;
    const int* ncenter; const double* xyz; const double* Z;
};

void os_1d(int la, int lb, double PA, double PB, double oo2p, std::vector<double>& S, int w) {
    // S(i,j) 1-D overlap recursion (without the common prefactor)
    S.assign((size_t)(la + 1) * w, 0.0);
    S[0] = 1.0;
    for (int i = 0; i <= la; ++i)
        for (int j = 0; j <= lb; ++j) {
            if (i == 0 && j == 0) continue;
            double v;
            if (i > 0) {
                v = PA * S[(i - 1) * w + j];
                if (i > 1) v += (i - 1) * oo2p * S[(i - 2) * w + j];
                if (j > 0) v += j * oo2p * S[(i - 1) * w + j - 1];
            } else {
                v = PB * S[i * w + j - 1];
                if (j > 1) v += (j - 1) * oo2p * S[i * w + j - 2];
            }
            S[i * w + j] = v;
        }
}

}  // namespace

// =========================================================================== C ABI
extern "C" {

struct OracleHandle {
    Basis B;
};

void* orc_create(int natom, const double* xyz, int nshell, int nbasis, int jbasis,
                 const int* kstart, const int* katom, const int* ktype, const int* kprim,
                 const int* ksumtype, const int* qstart, const int* qfinal,
                 const int* qsbasis, const int* qfbasis, const double* gccoeff,
                 const double* gcexpo, const double* cons, const int* klmn) {
    static bool inited = false;
    if (!inited) { init_cart(); init_boys(); inited = true; }
    OracleHandle* h = new OracleHandle();
    Basis& B = h->B;
    B.natom = natom; B.nshell = nshell; B.nbasis = nbasis; B.jbasis = jbasis;
    B.xyz.assign(xyz, xyz + 3 * natom);
    B.kstart.assign(kstart, kstart + nshell); B.katom.assign(katom, katom + nshell);
    B.ktype.assign(ktype, ktype + nshell); B.kprim.assign(kprim, kprim + nshell);
    B.ksumtype.assign(ksumtype, ksumtype + nshell + 1);
    B.qstart.assign(qstart, qstart + nshell); B.qfinal.assign(qfinal, qfinal + nshell);
    B.qsbasis.assign(qsbasis, qsbasis + 4 * nshell); B.qfbasis.assign(qfbasis, qfbasis + 4 * nshell);
    B.gccoeff.assign(gccoeff, gccoeff + (size_t)MAXPRIM * nbasis);
    B.gcexpo.assign(gcexpo, gcexpo + (size_t)MAXPRIM * nbasis);
    B.cons.assign(cons, cons + nbasis);
    B.klmn.assign(klmn, klmn + 3 * nbasis);
    precompute(B);
    return h;
}

void orc_destroy(void* h) { delete (OracleHandle*)h; }

// Select the Boys function of the integral code: bit 0 = QUICK's fmt.f90 (else
// accurate), bit 1 = its exp(-X) one ulp up (the sensitivity probe); returns the
// previous mode.  Process-wide: set it before a build, not during one.
int orc_set_boys_mode(int mode) {
    const int old = g_boys_mode | (g_exp_ulp << 1);
    g_boys_mode = mode & 1;
    g_exp_ulp = (mode >> 1) & 1;
    return old;
}

void orc_boys(int M, double T, double* F) {
    static bool inited = false;
    if (!inited) { init_cart(); init_boys(); inited = true; }
    boys(M, T, F);
}

// Ycutoff (nshell x nshell) and cutprim (jbasis x jbasis), column-major.
void orc_schwarz(void* hv, double* Ycutoff, double* cutprim, int nthreads) {
    Basis& B = ((OracleHandle*)hv)->B;
    std::fill(Ycutoff, Ycutoff + (size_t)B.nshell * B.nshell, 0.0);
    std::fill(cutprim, cutprim + (size_t)B.jbasis * B.jbasis, 0.0);
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
#pragma omp parallel
    {
        Work W;
#pragma omp for schedule(dynamic, 1)
        for (int II = 0; II < B.nshell; ++II)
            for (int JJ = II; JJ < B.nshell; ++JJ) shell_cutoff(B, W, II, JJ, Ycutoff, cutprim);
    }
}

// cutmatrix(II,JJ) = max |D(j,i)| over the functions of shells II, JJ (cutoff.fh:16-92)
void orc_density_cutoff(void* hv, const double* dense, double* cutmatrix) {
    Basis& B = ((OracleHandle*)hv)->B;
    int n = B.nbasis, ns = B.nshell;
    for (int II = 0; II < ns; ++II)
        for (int JJ = II; JJ < ns; ++JJ) {
            double dn = 0.0;
            int i1 = B.ksumtype[II] + B.qs(II, B.qstart[II]), i2 = B.ksumtype[II] + B.qf(II, B.qfinal[II]);
            int j1 = B.ksumtype[JJ] + B.qs(JJ, B.qstart[JJ]), j2 = B.ksumtype[JJ] + B.qf(JJ, B.qfinal[JJ]);
            for (int i = i1; i <= i2; ++i)
                for (int j = j1; j <= j2; ++j) dn = std::max(dn, std::fabs(dense[(size_t)(j - 1) + (size_t)n * (i - 1)]));
            cutmatrix[II + (size_t)ns * JJ] = dn;
            cutmatrix[JJ + (size_t)ns * II] = dn;
        }
}

// o += G(dense) for the screened quartet set; returns the number of shell
// quartets evaluated.  Bra shells II = ii_begin, ii_begin + ii_stride, ... < ii_end
// only (a bounded sample when the range is partial).  nthreads <= 0 uses the
// OpenMP default.
long long get2e_core(void* hv, const double* dense, const double* dense_k, const double* cutmatrix,
                     const double* Ycutoff, const double* cutprim, double integralCutoff, double primLimit, double* o,
                     int ii_begin, int ii_end, int nthreads, int ii_stride, int gpu_screens);

long long orc_get2e(void* hv, const double* dense, const double* cutmatrix, const double* Ycutoff,
                    const double* cutprim, double integralCutoff, double primLimit, double* o,
                    int ii_begin, int ii_end, int nthreads, int ii_stride, int gpu_screens) {
    return get2e_core(hv, dense, nullptr, cutmatrix, Ycutoff, cutprim, integralCutoff, primLimit, o, ii_begin,
                      ii_end, nthreads, ii_stride, gpu_screens);
}

// Open-shell (UHF) build, get_oshell_eri (src/modules/include/eri.fh under OSHELL):
// oa += J[Da + Db] - K[Da], ob += J[Da + Db] - K[Db] on the quartets the open-shell
// density screen `cutmatrix` admits.  Each matrix is the closed-shell digestion with
// J read from Da + Db and K from 2 Da (2 Db).  Returns the quartets evaluated.
long long orc_get2e_uhf(void* hv, const double* Da, const double* Db, const double* cutmatrix,
                        const double* Ycutoff, const double* cutprim, double integralCutoff, double primLimit,
                        double* oa, double* ob, int nthreads) {
    Basis& B = ((OracleHandle*)hv)->B;
    const size_t nn = (size_t)B.nbasis * B.nbasis;
    std::vector<double> Dt(nn), Ka(nn), Kb(nn);
    for (size_t i = 0; i < nn; ++i) {
        Dt[i] = Da[i] + Db[i];
        Ka[i] = 2.0 * Da[i];
        Kb[i] = 2.0 * Db[i];
    }
    long long nq = get2e_core(hv, Dt.data(), Ka.data(), cutmatrix, Ycutoff, cutprim, integralCutoff, primLimit, oa, 0,
                              0, nthreads, 1, 0);
    get2e_core(hv, Dt.data(), Kb.data(), cutmatrix, Ycutoff, cutprim, integralCutoff, primLimit, ob, 0, 0, nthreads, 1, 0);
    return nq;
}

// QUICK's open-shell density screen (oshell_density_cutoff, src/modules/include/cutoff.fh:15-92):
// per shell pair the largest of |Da + Db|, |Da|, |Db| over its block.
void orc_density_cutoff_uhf(void* hv, const double* Da, const double* Db, double* cutmatrix) {
    Basis& B = ((OracleHandle*)hv)->B;
    int n = B.nbasis, ns = B.nshell;
    for (int II = 0; II < ns; ++II)
        for (int JJ = II; JJ < ns; ++JJ) {
            double dn = 0.0;
            int i1 = B.ksumtype[II] + B.qs(II, B.qstart[II]), i2 = B.ksumtype[II] + B.qf(II, B.qfinal[II]);
            int j1 = B.ksumtype[JJ] + B.qs(JJ, B.qstart[JJ]), j2 = B.ksumtype[JJ] + B.qf(JJ, B.qfinal[JJ]);
            for (int i = i1; i <= i2; ++i)
                for (int j = j1; j <= j2; ++j) {
                    const size_t k = (size_t)(j - 1) + (size_t)n * (i - 1);
                    dn = std::max({dn, std::fabs(Da[k] + Db[k]), std::fabs(Da[k]), std::fabs(Db[k])});
                }
            cutmatrix[II + (size_t)ns * JJ] = dn;
            cutmatrix[JJ + (size_t)ns * II] = dn;
        }
}

long long get2e_core(void* hv, const double* dense, const double* dense_k, const double* cutmatrix,
                     const double* Ycutoff, const double* cutprim, double integralCutoff, double primLimit, double* o,
                     int ii_begin, int ii_end, int nthreads, int ii_stride, int gpu_screens) {
    Basis& B = ((OracleHandle*)hv)->B;
    int n = B.nbasis, ns = B.nshell;
    if (ii_end <= 0 || ii_end > ns) ii_end = ns;
    if (ii_stride <= 0) ii_stride = 1;
    const int nII = (ii_end - ii_begin + ii_stride - 1) / ii_stride;
    Ctx C{&B, dense, cutmatrix, cutprim, integralCutoff, primLimit};
    C.dense_k = dense_k;
    C.gpu_screens = gpu_screens != 0;
    const double pair_cut = C.gpu_screens ? 1e-10 : -1.0;
    std::vector<double> G((size_t)n * n, 0.0);
    long long nq = 0;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
#pragma omp parallel reduction(+ : nq)
    {
        Work W;
        std::vector<double> Gt((size_t)n * n, 0.0);
#pragma omp for schedule(dynamic, 1) nowait
        for (int t = 0; t < nII; ++t) {
            const int II = ii_begin + t * ii_stride;
            for (int JJ = II; JJ < ns; ++JJ) {
                double t = Ycutoff[II + (size_t)ns * JJ];
                if (!(t > pair_cut)) continue;
                for (int KK = II; KK < ns; ++KK)
                    for (int LL = KK; LL < ns; ++LL) {
                        if (!(Ycutoff[KK + (size_t)ns * LL] > pair_cut)) continue;
                        double ct = t * Ycutoff[KK + (size_t)ns * LL];
                        if (!(ct > integralCutoff)) continue;
                        double dnmax = dnmax_of(C, II, JJ, KK, LL);
                        if (!(ct * dnmax > integralCutoff)) continue;
                        cshell_quartet(C, W, II, JJ, KK, LL, dnmax, Gt.data());
                        ++nq;
                    }
            }
        }
#pragma omp critical
        for (size_t i = 0; i < G.size(); ++i) G[i] += Gt[i];
    }
    // copySym: upper triangle takes the lower one
    for (int i = 0; i < n; ++i)
        for (int j = i + 1; j < n; ++j) G[(size_t)i + (size_t)n * j] = G[(size_t)j + (size_t)n * i];
    for (size_t i = 0; i < G.size(); ++i) o[i] += G[i];
    return nq;
}

// Overlap S, kinetic T and nuclear attraction V (nbasis^2, column-major).
// Z/xyz: point charges (nuclei, optionally followed by external charges).
void orc_oei(int nbasis, int maxcontract, const int* ncontract, const int* itype,
             const double* aexp, const double* dcoeff, const int* ncenter,
             const double* atom_xyz, int ncharge, const double* charge_xyz, const double* charge,
             double* S, double* Tk, double* V) {
    static bool inited = false;
    if (!inited) { init_cart(); init_boys(); inited = true; }
    std::vector<double> Sx, Sy, Sz;
    for (int mu = 0; mu < nbasis; ++mu)
        for (int nu = 0; nu <= mu; ++nu) {
            const int* a = &itype[3 * mu];
            const int* b = &itype[3 * nu];
            const double* A = &atom_xyz[3 * (ncenter[mu] - 1)];
            const double* Bc = &atom_xyz[3 * (ncenter[nu] - 1)];
            double s = 0.0, t = 0.0, v = 0.0;
            for (int p = 0; p < ncontract[mu]; ++p)
                for (int q = 0; q < ncontract[nu]; ++q) {
                    double al = aexp[p + maxcontract * mu], be = aexp[q + maxcontract * nu];
                    double cc = dcoeff[p + maxcontract * mu] * dcoeff[q + maxcontract * nu];
                    double zeta = al + be, oo2p = 0.5 / zeta;
                    double P[3], PA[3], PB[3], ab2 = 0.0;
                    for (int k = 0; k < 3; ++k) {
                        P[k] = (al * A[k] + be * Bc[k]) / zeta;
                        PA[k] = P[k] - A[k]; PB[k] = P[k] - Bc[k];
                        ab2 += (A[k] - Bc[k]) * (A[k] - Bc[k]);
                    }
                    double pre = std::exp(-al * be / zeta * ab2) * std::pow(PI / zeta, 1.5);
                    int w = b[0] + b[1] + b[2] + 3;
                    int la = a[0] + a[1] + a[2] + 2;
                    std::vector<double>* Sd[3] = {&Sx, &Sy, &Sz};
                    for (int k = 0; k < 3; ++k) os_1d(la, w - 1, PA[k], PB[k], oo2p, *Sd[k], w);
                    auto s1 = [&](int k, int i, int j) -> double {
                        if (i < 0 || j < 0) return 0.0;
                        return (*Sd[k])[i * w + j];
                    };
                    double sx = s1(0, a[0], b[0]), sy = s1(1, a[1], b[1]), sz = s1(2, a[2], b[2]);
                    s += cc * pre * sx * sy * sz;
                    // kinetic: T = sum_k T1d_k * prod_{other} S1d
                    auto t1 = [&](int k, int i, int j) -> double {
                        return 0.5 * (i * j * s1(k, i - 1, j - 1) + 4.0 * al * be * s1(k, i + 1, j + 1)
                                      - 2.0 * al * j * s1(k, i + 1, j - 1) - 2.0 * be * i * s1(k, i - 1, j + 1));
                    };
                    double tt = t1(0, a[0], b[0]) * sy * sz + sx * t1(1, a[1], b[1]) * sz + sx * sy * t1(2, a[2], b[2]);
                    t += cc * pre * tt;
                    // nuclear attraction via OS recursion with auxiliary index m
                    int L = a[0] + a[1] + a[2] + b[0] + b[1] + b[2];
                    for (int c = 0; c < ncharge; ++c) {
                        const double* Cc = &charge_xyz[3 * c];
                        double PC[3], pc2 = 0.0;
                        for (int k = 0; k < 3; ++k) { PC[k] = P[k] - Cc[k]; pc2 += PC[k] * PC[k]; }
                        double F[2 * LMAX_SIDE + 4];
                        boys(L, zeta * pc2, F);
                        // Obara-Saika recursion over (a, b, m), downward on a then b
                        struct Rec {
                            const double *PA, *PB, *PC; double oo2p; const double* F;
                            double operator()(int ax, int ay, int az, int bx, int by, int bz, int m) const {
                                if (ax < 0 || ay < 0 || az < 0 || bx < 0 || by < 0 || bz < 0) return 0.0;
                                if (ax + ay + az + bx + by + bz == 0) return F[m];
                                int bn[3] = {bx, by, bz};
                                if (ax + ay + az > 0) {
                                    int i = ax ? 0 : (ay ? 1 : 2);
                                    int a1[3] = {ax, ay, az}; a1[i]--;
                                    double r = PA[i] * (*this)(a1[0], a1[1], a1[2], bx, by, bz, m)
                                             - PC[i] * (*this)(a1[0], a1[1], a1[2], bx, by, bz, m + 1);
                                    if (a1[i] > 0) {
                                        int a2[3] = {a1[0], a1[1], a1[2]}; a2[i]--;
                                        r += a1[i] * oo2p * ((*this)(a2[0], a2[1], a2[2], bx, by, bz, m)
                                                            - (*this)(a2[0], a2[1], a2[2], bx, by, bz, m + 1));
                                    }
                                    if (bn[i] > 0) {
                                        int b1[3] = {bx, by, bz}; b1[i]--;
                                        r += bn[i] * oo2p * ((*this)(a1[0], a1[1], a1[2], b1[0], b1[1], b1[2], m)
                                                            - (*this)(a1[0], a1[1], a1[2], b1[0], b1[1], b1[2], m + 1));
                                    }
                                    return r;
                                }
                                int i = bx ? 0 : (by ? 1 : 2);
                                int b1[3] = {bx, by, bz}; b1[i]--;
                                double r = PB[i] * (*this)(0, 0, 0, b1[0], b1[1], b1[2], m)
                                         - PC[i] * (*this)(0, 0, 0, b1[0], b1[1], b1[2], m + 1);
                                if (b1[i] > 0) {
                                    int b2[3] = {b1[0], b1[1], b1[2]}; b2[i]--;
                                    r += b1[i] * oo2p * ((*this)(0, 0, 0, b2[0], b2[1], b2[2], m)
                                                        - (*this)(0, 0, 0, b2[0], b2[1], b2[2], m + 1));
                                }
                                return r;
                            }
                        } rec{PA, PB, PC, oo2p, F};
                        double vv = rec(a[0], a[1], a[2], b[0], b[1], b[2], 0);
                        v += -charge[c] * cc * 2.0 * PI / zeta * std::exp(-al * be / zeta * ab2) * vv;
                    }
                }
            S[mu + (size_t)nbasis * nu] = S[nu + (size_t)nbasis * mu] = s;
            Tk[mu + (size_t)nbasis * nu] = Tk[nu + (size_t)nbasis * mu] = t;
            V[mu + (size_t)nbasis * nu] = V[nu + (size_t)nbasis * mu] = v;
        }
}

}  // extern "C"
