// or_math.hpp -- small dense FP64 linear algebra, b-basis, 3-D DFT for the oracle.
//
// TEST INFRASTRUCTURE ONLY (see evp_oracle.h).  Restates, in plain C++, the
// arithmetic of lsevpfft/src/tensor_functions.f90 and the LAPACK / FFTW calls
// the reference makes.  LAPACK and FFTW are third-party (unpinned versions,
// conda-forge per readme.txt:10-11); their published algorithms are restated:
//   dgetrf/dgetrs/dgesv/dgetri  -> LU with partial pivoting (first max |a|)
//   dgesvd (polar_dcmp)          -> polar factor by scaled Newton iteration
//                                   (Higham 1986); the factor is unique
//   dsyev (3x3)                  -> cyclic Jacobi, eigenvalues ascending
//   dgecon + dlacn2              -> Hager/Higham 1-norm estimator (Higham 1988)
//   FFTW C2C                     -> recursive mixed-radix Cooley-Tukey DFT
#pragma once
#include <cmath>
#include <complex>
#include <cstring>
#include <vector>
#include <algorithm>
#include <cfloat>

namespace orc {

typedef std::complex<double> cplx;
static const double PI = 4.0 * std::atan(1.0);  // global.f90:3
static const double TINY = DBL_MIN;              // tiny(1.0d0)
static const double HUGE_ = DBL_MAX;             // huge(1.0d0)

// b-basis constants (tensor_functions.f90:25-28; real(8) under -fdefault-real-8)
static const double RSQ2 = std::sqrt(2.0) / 2.0;
static const double RSQ3 = std::sqrt(3.0) / 3.0;
static const double RSQ6 = std::sqrt(6.0) / 6.0;
static const double RSQ23 = std::sqrt(2.0) * std::sqrt(3.0) / 3.0;

typedef double M3[3][3];
typedef double M6[6][6];
typedef double T4[3][3][3][3];

// ---------------------------------------------------------------- b-basis
// Basis tensors B(:,:,n) implied by CHG_BASIS (tensor_functions.f90:21-198).
struct BBasis {
    double b[6][3][3];
    int nnz[6];
    int ii[6][3], jj[6][3];
    double v[6][3];
    BBasis() {
        std::memset(b, 0, sizeof(b));
        b[0][0][0] = -RSQ2; b[0][1][1] = RSQ2;
        b[1][0][0] = -RSQ6; b[1][1][1] = -RSQ6; b[1][2][2] = RSQ23;
        b[2][1][2] = RSQ2;  b[2][2][1] = RSQ2;
        b[3][0][2] = RSQ2;  b[3][2][0] = RSQ2;
        b[4][0][1] = RSQ2;  b[4][1][0] = RSQ2;
        b[5][0][0] = RSQ3;  b[5][1][1] = RSQ3; b[5][2][2] = RSQ3;
        for (int n = 0; n < 6; n++) {
            nnz[n] = 0;
            for (int i = 0; i < 3; i++)
                for (int j = 0; j < 3; j++)
                    if (b[n][i][j] != 0.0) {
                        ii[n][nnz[n]] = i; jj[n][nnz[n]] = j; v[n][nnz[n]] = b[n][i][j];
                        nnz[n]++;
                    }
        }
    }
};
static const BBasis BB;

// CHG_BASIS iopt=2, kdim=6 (tensor_functions.f90:45-54)
inline void t2_to_b6(const M3 c, double ce[6]) {
    ce[0] = RSQ2 * c[1][1] - RSQ2 * c[0][0];
    ce[1] = RSQ23 * c[2][2] - RSQ6 * c[1][1] - RSQ6 * c[0][0];
    ce[2] = RSQ2 * c[1][2] + RSQ2 * c[2][1];
    ce[3] = RSQ2 * c[0][2] + RSQ2 * c[2][0];
    ce[4] = RSQ2 * c[0][1] + RSQ2 * c[1][0];
    ce[5] = RSQ3 * c[0][0] + RSQ3 * c[1][1] + RSQ3 * c[2][2];
}
// CHG_BASIS iopt=2, kdim=5
inline void t2_to_b5(const M3 c, double ce[5]) {
    ce[0] = RSQ2 * c[1][1] - RSQ2 * c[0][0];
    ce[1] = RSQ23 * c[2][2] - RSQ6 * c[1][1] - RSQ6 * c[0][0];
    ce[2] = RSQ2 * c[1][2] + RSQ2 * c[2][1];
    ce[3] = RSQ2 * c[0][2] + RSQ2 * c[2][0];
    ce[4] = RSQ2 * c[0][1] + RSQ2 * c[1][0];
}
// CHG_BASIS iopt=1, kdim=6 (tensor_functions.f90:37-41)
inline void b6_to_t2(const double ce[6], M3 c) {
    c[0][0] = RSQ3 * ce[5] - RSQ2 * ce[0] - RSQ6 * ce[1];
    c[0][1] = RSQ2 * ce[4];
    c[0][2] = RSQ2 * ce[3];
    c[1][0] = RSQ2 * ce[4];
    c[1][1] = RSQ3 * ce[5] + RSQ2 * ce[0] - RSQ6 * ce[1];
    c[1][2] = RSQ2 * ce[2];
    c[2][0] = RSQ2 * ce[3];
    c[2][1] = RSQ2 * ce[2];
    c[2][2] = RSQ3 * ce[5] + RSQ23 * ce[1];
}
// CHG_BASIS iopt=4: CE4(n,m) = B(:,:,n) : C4 : B(:,:,m)
inline void t4_to_b66(const T4 c, M6 ce) {
    for (int n = 0; n < 6; n++)
        for (int m = 0; m < 6; m++) {
            double s = 0.0;
            for (int p = 0; p < BB.nnz[n]; p++)
                for (int q = 0; q < BB.nnz[m]; q++)
                    s += BB.v[n][p] * BB.v[m][q] * c[BB.ii[n][p]][BB.jj[n][p]][BB.ii[m][q]][BB.jj[m][q]];
            ce[n][m] = s;
        }
}
// CHG_BASIS iopt=3: C4 = sum_nm CE4(n,m) B(n) (x) B(m)
inline void b66_to_t4(const M6 ce, T4 c) {
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            for (int k = 0; k < 3; k++)
                for (int l = 0; l < 3; l++) {
                    double s = 0.0;
                    for (int n = 0; n < 6; n++) {
                        double bn = BB.b[n][i][j];
                        if (bn == 0.0) continue;
                        for (int m = 0; m < 6; m++) {
                            double bm = BB.b[m][k][l];
                            if (bm == 0.0) continue;
                            s += ce[n][m] * bn * bm;
                        }
                    }
                    c[i][j][k][l] = s;
                }
}

// VOIGT_VPSC (tensor_functions.f90:208-261), IJV = 11,22,33,23,13,12
static const int IJV[6][2] = {{0, 0}, {1, 1}, {2, 2}, {1, 2}, {0, 2}, {0, 1}};
inline void voigt_to_t2(const double t1[6], M3 t2) {
    for (int i = 0; i < 6; i++) { t2[IJV[i][0]][IJV[i][1]] = t1[i]; t2[IJV[i][1]][IJV[i][0]] = t1[i]; }
}
inline void t2_to_voigt(const M3 t2, double t1[6]) {
    for (int i = 0; i < 6; i++) t1[i] = t2[IJV[i][0]][IJV[i][1]];
}
inline void v66_to_t4(const M6 c2, T4 c4) {
    for (int i = 0; i < 6; i++)
        for (int j = 0; j < 6; j++) {
            int i1 = IJV[i][0], i2 = IJV[i][1], j1 = IJV[j][0], j2 = IJV[j][1];
            c4[i1][i2][j1][j2] = c2[i][j]; c4[i2][i1][j1][j2] = c2[i][j];
            c4[i1][i2][j2][j1] = c2[i][j]; c4[i2][i1][j2][j1] = c2[i][j];
        }
}
inline void t4_to_v66(const T4 c4, M6 c2) {
    for (int i = 0; i < 6; i++)
        for (int j = 0; j < 6; j++) c2[i][j] = c4[IJV[i][0]][IJV[i][1]][IJV[j][0]][IJV[j][1]];
}

// vm_stress / vm_strain (tensor_functions.f90:266-289)
inline double vm_stress(const M3 d) {
    double h = (d[0][0] + d[1][1] + d[2][2]) / 3.0;
    return std::sqrt(3.0 / 2.0 * ((d[0][0] - h) * (d[0][0] - h) + (d[1][1] - h) * (d[1][1] - h) + (d[2][2] - h) * (d[2][2] - h) +
                                  d[0][1] * d[0][1] + d[0][2] * d[0][2] + d[1][2] * d[1][2] + d[1][0] * d[1][0] +
                                  d[2][0] * d[2][0] + d[2][1] * d[2][1]));
}
inline double vm_strain(const M3 d) {
    double h = (d[0][0] + d[1][1] + d[2][2]) / 3.0;
    return std::sqrt(2.0 / 3.0 * ((d[0][0] - h) * (d[0][0] - h) + (d[1][1] - h) * (d[1][1] - h) + (d[2][2] - h) * (d[2][2] - h) +
                                  d[0][1] * d[0][1] + d[0][2] * d[0][2] + d[1][2] * d[1][2] + d[1][0] * d[1][0] +
                                  d[2][0] * d[2][0] + d[2][1] * d[2][1]));
}
inline void sym33(const M3 a, M3 s) {
    s[0][0] = a[0][0]; s[1][1] = a[1][1]; s[2][2] = a[2][2];
    s[0][1] = 0.5 * (a[0][1] + a[1][0]); s[0][2] = 0.5 * (a[0][2] + a[2][0]); s[1][2] = 0.5 * (a[1][2] + a[2][1]);
    s[1][0] = s[0][1]; s[2][0] = s[0][2]; s[2][1] = s[1][2];
}
inline void antisym33(const M3 a, M3 s) {
    s[0][0] = s[1][1] = s[2][2] = 0.0;
    s[0][1] = 0.5 * (a[0][1] - a[1][0]); s[0][2] = 0.5 * (a[0][2] - a[2][0]); s[1][2] = 0.5 * (a[1][2] - a[2][1]);
    s[1][0] = -s[0][1]; s[2][0] = -s[0][2]; s[2][1] = -s[1][2];
}
// determinant33 (tensor_functions.f90:442-456)
inline double det33(const M3 m) {
    return m[0][0] * m[1][1] * m[2][2] + m[0][1] * m[1][2] * m[2][0] + m[0][2] * m[1][0] * m[2][1] -
           m[2][0] * m[1][1] * m[0][2] - m[2][1] * m[1][2] * m[0][0] - m[2][2] * m[1][0] * m[0][1];
}
// determinant33 of types.f90:751-756 (cofactor form, used by diagnostics)
inline double det33_cof(const M3 a) {
    return a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) - a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]) +
           a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
}
inline void matmul3(const M3 a, const M3 b, M3 c) {
    M3 t;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double s = 0.0;
            for (int k = 0; k < 3; k++) s += a[i][k] * b[k][j];
            t[i][j] = s;
        }
    std::memcpy(c, t, sizeof(t));
}
inline void transpose3(const M3 a, M3 t) {
    M3 r;
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) r[i][j] = a[j][i];
    std::memcpy(t, r, sizeof(r));
}
inline void copy3(const M3 a, M3 b) { std::memcpy(b, a, sizeof(M3)); }
inline void eye3(M3 a) { for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) a[i][j] = (i == j) ? 1.0 : 0.0; }
inline double frob3(const M3 a) { double s = 0; for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) s += a[i][j] * a[i][j]; return std::sqrt(s); }
inline double norm2v(const double* v, int n) { double s = 0; for (int i = 0; i < n; i++) s += v[i] * v[i]; return std::sqrt(s); }

// euler(iopt=2) (tensor_functions.f90:550-566)
inline void euler2(double ph, double th, double tm, M3 a) {
    double sph = std::sin(ph), cph = std::cos(ph), sth = std::sin(th), cth = std::cos(th), stm = std::sin(tm), ctm = std::cos(tm);
    a[0][0] = ctm * cph - sph * stm * cth;
    a[1][0] = -stm * cph - sph * ctm * cth;
    a[2][0] = sph * sth;
    a[0][1] = ctm * sph + cph * stm * cth;
    a[1][1] = -sph * stm + cph * ctm * cth;
    a[2][1] = -sth * cph;
    a[0][2] = sth * stm;
    a[1][2] = ctm * sth;
    a[2][2] = cth;
}

// ---------------------------------------------------------------- LU (LAPACK dgetrf / dgesv / dgetri)
// a: row-major n x n, a[i*n+j] = A(i,j).  Returns LAPACK-style info (0 ok, k>0: U(k,k) == 0).
inline int lu_factor(double* a, int n, int* piv) {
    int info = 0;
    for (int k = 0; k < n; k++) {
        int p = k;
        double amax = std::fabs(a[k * n + k]);
        for (int i = k + 1; i < n; i++)
            if (std::fabs(a[i * n + k]) > amax) { amax = std::fabs(a[i * n + k]); p = i; }
        piv[k] = p;
        if (a[p * n + k] != 0.0) {
            if (p != k)
                for (int j = 0; j < n; j++) std::swap(a[k * n + j], a[p * n + j]);
            double r = 1.0 / a[k * n + k];
            for (int i = k + 1; i < n; i++) a[i * n + k] *= r;
        } else if (info == 0) {
            info = k + 1;
        }
        for (int i = k + 1; i < n; i++) {
            double l = a[i * n + k];
            if (l != 0.0)
                for (int j = k + 1; j < n; j++) a[i * n + j] -= l * a[k * n + j];
        }
    }
    return info;
}
inline void lu_solve(const double* lu, int n, const int* piv, double* b) {
    for (int k = 0; k < n; k++)
        if (piv[k] != k) std::swap(b[k], b[piv[k]]);
    for (int i = 0; i < n; i++) {
        double s = b[i];
        for (int j = 0; j < i; j++) s -= lu[i * n + j] * b[j];
        b[i] = s;
    }
    for (int i = n - 1; i >= 0; i--) {
        double s = b[i];
        for (int j = i + 1; j < n; j++) s -= lu[i * n + j] * b[j];
        b[i] = s / lu[i * n + i];
    }
}
// lu_inverse (tensor_functions.f90:313-337): returns info (nonzero = singular).
inline int lu_inverse(double* a, int n) {
    double lu[36];
    int piv[6];
    std::memcpy(lu, a, sizeof(double) * n * n);
    int info = lu_factor(lu, n, piv);
    if (info != 0) return info;
    for (int c = 0; c < n; c++) {
        double col[6];
        for (int i = 0; i < n; i++) col[i] = (i == c) ? 1.0 : 0.0;
        lu_solve(lu, n, piv, col);
        for (int i = 0; i < n; i++) a[i * n + c] = col[i];
    }
    return 0;
}
// lu_eqsystem (tensor_functions.f90:344-359): b <- A^{-1} b; returns info.
inline int lu_eqsystem(double* a, double* b, int n) {
    int piv[6];
    int info = lu_factor(a, n, piv);
    if (info != 0) return info;
    lu_solve(a, n, piv, b);
    return 0;
}
inline int inv3(const M3 a, M3 ainv) {
    double t[9];
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) t[i * 3 + j] = a[i][j];
    int info = lu_inverse(t, 3);
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) ainv[i][j] = t[i * 3 + j];
    return info;
}
inline int inv6(const M6 a, M6 ainv) {
    double t[36];
    for (int i = 0; i < 6; i++) for (int j = 0; j < 6; j++) t[i * 6 + j] = a[i][j];
    int info = lu_inverse(t, 6);
    for (int i = 0; i < 6; i++) for (int j = 0; j < 6; j++) ainv[i][j] = t[i * 6 + j];
    return info;
}

// ---------------------------------------------------------------- polar decomposition (polar_dcmp)
// F = R U.  Scaled Newton iteration X <- (g X + X^{-T}/g)/2 (Higham 1986).
inline void adj_inv3(const M3 a, M3 inv) {
    double c00 = a[1][1] * a[2][2] - a[1][2] * a[2][1];
    double c01 = a[1][2] * a[2][0] - a[1][0] * a[2][2];
    double c02 = a[1][0] * a[2][1] - a[1][1] * a[2][0];
    double det = a[0][0] * c00 + a[0][1] * c01 + a[0][2] * c02;
    double r = 1.0 / det;
    inv[0][0] = c00 * r; inv[1][0] = c01 * r; inv[2][0] = c02 * r;
    inv[0][1] = (a[0][2] * a[2][1] - a[0][1] * a[2][2]) * r;
    inv[1][1] = (a[0][0] * a[2][2] - a[0][2] * a[2][0]) * r;
    inv[2][1] = (a[0][1] * a[2][0] - a[0][0] * a[2][1]) * r;
    inv[0][2] = (a[0][1] * a[1][2] - a[0][2] * a[1][1]) * r;
    inv[1][2] = (a[0][2] * a[1][0] - a[0][0] * a[1][2]) * r;
    inv[2][2] = (a[0][0] * a[1][1] - a[0][1] * a[1][0]) * r;
}
inline void polar(const M3 F, M3 R, M3 U) {
    M3 X, Xi, Xn;
    copy3(F, X);
    bool scale = true;
    for (int it = 0; it < 60; it++) {
        adj_inv3(X, Xi);
        double g = 1.0;
        if (scale) g = std::sqrt(frob3(Xi) / frob3(X));
        double d = 0.0, nn = 0.0;
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) {
                Xn[i][j] = 0.5 * (g * X[i][j] + Xi[j][i] / g);
                d += (Xn[i][j] - X[i][j]) * (Xn[i][j] - X[i][j]);
                nn += Xn[i][j] * Xn[i][j];
            }
        copy3(Xn, X);
        if (d <= 1e-20 * nn) scale = false;
        if (d <= 1e-30 * nn) break;
    }
    copy3(X, R);
    M3 Rt, Ut;
    transpose3(R, Rt);
    matmul3(Rt, F, Ut);
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) U[i][j] = 0.5 * (Ut[i][j] + Ut[j][i]);
}

// ---------------------------------------------------------------- symmetric 3x3 eigen (dsyev 'V','U')
inline void sym_eig3(const M3 A, double w[3], M3 Q) {
    double a[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) a[i][j] = (i <= j) ? A[i][j] : A[j][i];
    eye3(Q);
    for (int sweep = 0; sweep < 60; sweep++) {
        double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
        if (off == 0.0) break;
        double diag = a[0][0] * a[0][0] + a[1][1] * a[1][1] + a[2][2] * a[2][2];
        if (off < 1e-36 * diag) break;
        for (int p = 0; p < 2; p++)
            for (int q = p + 1; q < 3; q++) {
                if (a[p][q] == 0.0) continue;
                double theta = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
                double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < 3; k++) {
                    double akp = a[k][p], akq = a[k][q];
                    a[k][p] = c * akp - s * akq;
                    a[k][q] = s * akp + c * akq;
                }
                for (int k = 0; k < 3; k++) {
                    double apk = a[p][k], aqk = a[q][k];
                    a[p][k] = c * apk - s * aqk;
                    a[q][k] = s * apk + c * aqk;
                }
                for (int k = 0; k < 3; k++) {
                    double qkp = Q[k][p], qkq = Q[k][q];
                    Q[k][p] = c * qkp - s * qkq;
                    Q[k][q] = s * qkp + c * qkq;
                }
            }
    }
    int idx[3] = {0, 1, 2};
    double d[3] = {a[0][0], a[1][1], a[2][2]};
    std::sort(idx, idx + 3, [&](int x, int y) { return d[x] < d[y]; });
    M3 Qs;
    for (int c = 0; c < 3; c++) {
        w[c] = d[idx[c]];
        for (int r = 0; r < 3; r++) Qs[r][c] = Q[r][idx[c]];
    }
    copy3(Qs, Q);
}

// ---------------------------------------------------------------- 1-norm condition estimate (dgetrf + dgecon)
// dlacn2 reverse-communication estimator restated as a loop (Higham 1988, Alg. 4.1).
inline double cond1_est_6x6(const M6 Ain) {
    const int n = 6;
    double lu[36];
    int piv[6];
    double anorm = 0.0;
    for (int j = 0; j < n; j++) {
        double cs = 0.0;
        for (int i = 0; i < n; i++) cs += std::fabs(Ain[i][j]);
        anorm = std::max(anorm, cs);
    }
    for (int i = 0; i < n; i++) for (int j = 0; j < n; j++) lu[i * n + j] = Ain[i][j];
    if (lu_factor(lu, n, piv) != 0) return HUGE_;
    // x <- inv(U) inv(L) x   (kase 1)  /  x <- inv(L^T) inv(U^T) x  (kase 2); no row permutation (dgecon)
    auto solveA = [&](double* x) {
        for (int i = 0; i < n; i++) { double s = x[i]; for (int j = 0; j < i; j++) s -= lu[i * n + j] * x[j]; x[i] = s; }
        for (int i = n - 1; i >= 0; i--) { double s = x[i]; for (int j = i + 1; j < n; j++) s -= lu[i * n + j] * x[j]; x[i] = s / lu[i * n + i]; }
    };
    auto solveAT = [&](double* x) {
        for (int i = 0; i < n; i++) { double s = x[i]; for (int j = 0; j < i; j++) s -= lu[j * n + i] * x[j]; x[i] = s / lu[i * n + i]; }
        for (int i = n - 1; i >= 0; i--) { double s = x[i]; for (int j = i + 1; j < n; j++) s -= lu[j * n + i] * x[j]; x[i] = s; }
    };
    auto dasum = [&](const double* x) { double s = 0; for (int i = 0; i < n; i++) s += std::fabs(x[i]); return s; };
    auto idamax = [&](const double* x) { int k = 0; double m = std::fabs(x[0]); for (int i = 1; i < n; i++) if (std::fabs(x[i]) > m) { m = std::fabs(x[i]); k = i; } return k; };
    double x[6], v[6];
    int isgn[6];
    const int ITMAX = 5;
    for (int i = 0; i < n; i++) x[i] = 1.0 / n;
    solveA(x);
    double est = dasum(x);
    for (int i = 0; i < n; i++) { x[i] = (x[i] >= 0.0) ? 1.0 : -1.0; isgn[i] = (int)std::lround(x[i]); }
    solveAT(x);
    int j = idamax(x);
    int iter = 2;
    while (true) {
        for (int i = 0; i < n; i++) x[i] = 0.0;
        x[j] = 1.0;
        solveA(x);
        std::memcpy(v, x, sizeof(v));
        double estold = est;
        est = dasum(v);
        bool changed = false;
        for (int i = 0; i < n; i++) {
            double xs = (x[i] >= 0.0) ? 1.0 : -1.0;
            if ((int)std::lround(xs) != isgn[i]) { changed = true; break; }
        }
        if (!changed) break;
        if (est <= estold) break;
        for (int i = 0; i < n; i++) { x[i] = (x[i] >= 0.0) ? 1.0 : -1.0; isgn[i] = (int)std::lround(x[i]); }
        solveAT(x);
        int jlast = j;
        j = idamax(x);
        if ((x[jlast] != std::fabs(x[j])) && (iter < ITMAX)) { iter++; continue; }
        break;
    }
    double altsgn = 1.0;
    for (int i = 0; i < n; i++) { x[i] = altsgn * (1.0 + (double)i / (double)(n - 1)); altsgn = -altsgn; }
    solveA(x);
    double temp = 2.0 * (dasum(x) / (double)(3 * n));
    if (temp > est) est = temp;
    double ainvnm = est;
    if (ainvnm == 0.0) return HUGE_;
    double rcond = (1.0 / ainvnm) / anorm;
    if (!(rcond > 0.0)) return HUGE_;
    return 1.0 / rcond;
}

// ---------------------------------------------------------------- matrix exponential (various_functions.f90:1829-1967)
inline double l1_norm33(const M3 m) {
    double l1 = 0.0;
    for (int j = 0; j < 3; j++) {
        double cs = std::fabs(m[0][j]) + std::fabs(m[1][j]) + std::fabs(m[2][j]);
        if (cs > l1) l1 = cs;
    }
    return l1;
}
inline void expm_taylor3(const M3 a, M3 e) {
    M3 a2, a3;
    matmul3(a, a, a2);
    matmul3(a2, a, a3);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) e[i][j] = (i == j ? 1.0 : 0.0) + a[i][j] + a2[i][j] / 2.0 + a3[i][j] / 6.0;
}
inline int expm_pade13(const M3 mat, M3 e) {
    const double theta13 = 5.371920351148152;
    const double b[14] = {64764752532480000.0, 32382376266240000.0, 7771770303897600.0, 1187353796428800.0,
                          129060195264000.0, 10559470521600.0, 670442572800.0, 33522128640.0, 1323241920.0,
                          40840800.0, 960960.0, 16380.0, 182.0, 1.0};
    M3 A;
    copy3(mat, A);
    double normA = l1_norm33(A);
    if (normA <= 0.0) { eye3(e); return 0; }
    if (!(normA < 1.0e300)) return -1;  // non-finite input
    int s = 0;
    if (normA > theta13) s = (int)std::ceil(std::log(normA / theta13) / std::log(2.0));
    double sc = std::pow(2.0, s);
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) A[i][j] = A[i][j] / sc;
    M3 A2, A4, A6, t1, t2, U, V;
    matmul3(A, A, A2); matmul3(A2, A2, A4); matmul3(A2, A4, A6);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) t1[i][j] = b[13] * A6[i][j] + b[11] * A4[i][j] + b[9] * A2[i][j];
    matmul3(A6, t1, t2);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) t2[i][j] = t2[i][j] + b[7] * A6[i][j] + b[5] * A4[i][j] + b[3] * A2[i][j] + b[1] * (i == j ? 1.0 : 0.0);
    matmul3(A, t2, U);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) t1[i][j] = b[12] * A6[i][j] + b[10] * A4[i][j] + b[8] * A2[i][j];
    matmul3(A6, t1, V);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) V[i][j] = V[i][j] + b[6] * A6[i][j] + b[4] * A4[i][j] + b[2] * A2[i][j] + b[0] * (i == j ? 1.0 : 0.0);
    double Q[9], X[3][3];
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) { Q[i * 3 + j] = V[i][j] - U[i][j]; X[i][j] = V[i][j] + U[i][j]; }
    int piv[3];
    int info = lu_factor(Q, 3, piv);
    if (info != 0) return info;
    for (int c = 0; c < 3; c++) {
        double col[3] = {X[0][c], X[1][c], X[2][c]};
        lu_solve(Q, 3, piv, col);
        for (int r = 0; r < 3; r++) e[r][c] = col[r];
    }
    for (int k = 0; k < s; k++) matmul3(e, e, e);
    return 0;
}
inline int expm_adaptive(const M3 m, M3 e) {
    if (l1_norm33(m) <= 1.0e-1) { expm_taylor3(m, e); return 0; }
    return expm_pade13(m, e);
}

// ---------------------------------------------------------------- DFT (FFTW_FORWARD = -1, unnormalised)
struct Fft1 {
    int n = 0;
    std::vector<int> fac;
    std::vector<cplx> w;  // w[e] = exp(sign 2 pi i e / n)
    int sign = -1;
    void init(int n_, int sign_) {
        n = n_; sign = sign_;
        fac.clear();
        int m = n;
        for (int p = 2; m > 1;) {
            if (m % p == 0) { fac.push_back(p); m /= p; }
            else p++;
        }
        w.resize(n);
        for (int e = 0; e < n; e++) {
            double ang = sign * 2.0 * PI * (double)e / (double)n;
            w[e] = cplx(std::cos(ang), std::sin(ang));
        }
    }
    // out[0..len) = DFT of in[0], in[stride], ...; fac_i indexes the factor list
    void rec(cplx* out, const cplx* in, int stride, int len, int fi) const {
        if (len == 1) { out[0] = in[0]; return; }
        int p = fac[fi], m = len / p;
        for (int r = 0; r < p; r++) rec(out + r * m, in + r * stride, stride * p, m, fi + 1);
        int tw = n / len;
        cplx t[16];
        for (int k = 0; k < m; k++) {
            for (int r = 0; r < p; r++) t[r] = out[r * m + k] * w[((long)r * k * tw) % n];
            for (int q = 0; q < p; q++) {
                cplx s(0.0, 0.0);
                for (int r = 0; r < p; r++) s += t[r] * w[((long)((r * q) % p) * (n / p)) % n];
                out[q * m + k] = s;
            }
        }
    }
    void run(cplx* x, cplx* scratch) const {
        if (n == 1) return;
        std::memcpy(scratch, x, sizeof(cplx) * n);
        rec(x, scratch, 1, n, 0);
    }
};

// In-place 3-D DFT of one field, layout x fastest.
inline void fft3_field(cplx* f, int n1, int n2, int n3, const Fft1& p1, const Fft1& p2, const Fft1& p3) {
    long nyz = (long)n2 * n3;
#pragma omp parallel
    {
        std::vector<cplx> line(std::max(n1, std::max(n2, n3))), scr(line.size());
#pragma omp for schedule(static)
        for (long r = 0; r < nyz; r++) {
            cplx* row = f + r * n1;
            p1.run(row, scr.data());
        }
#pragma omp for schedule(static)
        for (long r = 0; r < (long)n1 * n3; r++) {
            long i = r % n1, k = r / n1;
            for (int j = 0; j < n2; j++) line[j] = f[i + (long)n1 * (j + (long)n2 * k)];
            p2.run(line.data(), scr.data());
            for (int j = 0; j < n2; j++) f[i + (long)n1 * (j + (long)n2 * k)] = line[j];
        }
#pragma omp for schedule(static)
        for (long r = 0; r < (long)n1 * n2; r++) {
            for (int k = 0; k < n3; k++) line[k] = f[r + (long)n1 * n2 * k];
            p3.run(line.data(), scr.data());
            for (int k = 0; k < n3; k++) f[r + (long)n1 * n2 * k] = line[k];
        }
    }
}

}  // namespace orc
