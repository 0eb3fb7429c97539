// evp_math.cuh -- FP64 small-tensor arithmetic shared by the sm_100a kernels
// and the host-side serial tails of the LS-EVPFFT solve.
//
// Conventions: 3x3 tensors are double[9] row-major (a[3*i+j] = A(i,j));
// 6x6 matrices double[36] row-major; 4th-order tensors double[81] with
// index ((i*3+j)*3+k)*3+l.  "b6" vectors use the reference's orthonormal
// b-basis (5 deviatoric components + 1 hydrostatic; tensor_functions.f90:21-198).
#pragma once
#include <cmath>
#include <cfloat>

#if defined(__CUDACC__)
#define EVP_HD __host__ __device__ __forceinline__
#else
#define EVP_HD inline
#endif

namespace evp {

// b-basis constants (tensor_functions.f90:25-28; FP64 because the reference
// builds with -fdefault-real-8).
#define EVP_RSQ2 0.70710678118654757
#define EVP_RSQ3 0.5773502691896257
#define EVP_RSQ6 0.40824829046386296
#define EVP_RSQ23 0.8164965809277261
#define EVP_PI 3.1415926535897931
#define EVP_TINY 2.2250738585072014e-308
#define EVP_HUGE 1.7976931348623157e+308

// ---- CHG_BASIS iopt=2, kdim=6: 3x3 -> b6
EVP_HD void t2_to_b6(const double* c, double* ce) {
    ce[0] = EVP_RSQ2 * c[4] - EVP_RSQ2 * c[0];
    ce[1] = EVP_RSQ23 * c[8] - EVP_RSQ6 * c[4] - EVP_RSQ6 * c[0];
    ce[2] = EVP_RSQ2 * c[5] + EVP_RSQ2 * c[7];
    ce[3] = EVP_RSQ2 * c[2] + EVP_RSQ2 * c[6];
    ce[4] = EVP_RSQ2 * c[1] + EVP_RSQ2 * c[3];
    ce[5] = EVP_RSQ3 * c[0] + EVP_RSQ3 * c[4] + EVP_RSQ3 * c[8];
}
// symmetric 3x3 stored as s6 = (11,22,33,23,13,12) -> b6
EVP_HD void s6_to_b6(const double* s, double* ce) {
    ce[0] = EVP_RSQ2 * s[1] - EVP_RSQ2 * s[0];
    ce[1] = EVP_RSQ23 * s[2] - EVP_RSQ6 * s[1] - EVP_RSQ6 * s[0];
    ce[2] = EVP_RSQ2 * s[3] + EVP_RSQ2 * s[3];
    ce[3] = EVP_RSQ2 * s[4] + EVP_RSQ2 * s[4];
    ce[4] = EVP_RSQ2 * s[5] + EVP_RSQ2 * s[5];
    ce[5] = EVP_RSQ3 * s[0] + EVP_RSQ3 * s[1] + EVP_RSQ3 * s[2];
}
// CHG_BASIS iopt=2, kdim=5
EVP_HD void t2_to_b5(const double* c, double* ce) {
    ce[0] = EVP_RSQ2 * c[4] - EVP_RSQ2 * c[0];
    ce[1] = EVP_RSQ23 * c[8] - EVP_RSQ6 * c[4] - EVP_RSQ6 * c[0];
    ce[2] = EVP_RSQ2 * c[5] + EVP_RSQ2 * c[7];
    ce[3] = EVP_RSQ2 * c[2] + EVP_RSQ2 * c[6];
    ce[4] = EVP_RSQ2 * c[1] + EVP_RSQ2 * c[3];
}
// CHG_BASIS iopt=1, kdim=6: b6 -> symmetric 3x3 as s6 (11,22,33,23,13,12)
EVP_HD void b6_to_s6(const double* ce, double* s) {
    s[0] = EVP_RSQ3 * ce[5] - EVP_RSQ2 * ce[0] - EVP_RSQ6 * ce[1];
    s[1] = EVP_RSQ3 * ce[5] + EVP_RSQ2 * ce[0] - EVP_RSQ6 * ce[1];
    s[2] = EVP_RSQ3 * ce[5] + EVP_RSQ23 * ce[1];
    s[3] = EVP_RSQ2 * ce[2];
    s[4] = EVP_RSQ2 * ce[3];
    s[5] = EVP_RSQ2 * ce[4];
}
EVP_HD void s6_to_t2(const double* s, double* c) {
    c[0] = s[0]; c[4] = s[1]; c[8] = s[2];
    c[5] = c[7] = s[3];
    c[2] = c[6] = s[4];
    c[1] = c[3] = s[5];
}
EVP_HD void t2_to_s6(const double* c, double* s) {  // upper triangle
    s[0] = c[0]; s[1] = c[4]; s[2] = c[8]; s[3] = c[5]; s[4] = c[2]; s[5] = c[1];
}
EVP_HD void b6_to_t2(const double* ce, double* c) {
    double s[6];
    b6_to_s6(ce, s);
    s6_to_t2(s, c);
}

// Nonzeros of the basis tensors B(:,:,n): (flat index i*3+j, value)
struct BasisNZ { int n; int idx[3]; double v[3]; };
EVP_HD BasisNZ basis_nz(int n) {
    BasisNZ b;
    switch (n) {
        case 0: b.n = 2; b.idx[0] = 0; b.v[0] = -EVP_RSQ2; b.idx[1] = 4; b.v[1] = EVP_RSQ2; break;
        case 1: b.n = 3; b.idx[0] = 0; b.v[0] = -EVP_RSQ6; b.idx[1] = 4; b.v[1] = -EVP_RSQ6; b.idx[2] = 8; b.v[2] = EVP_RSQ23; break;
        case 2: b.n = 2; b.idx[0] = 5; b.v[0] = EVP_RSQ2; b.idx[1] = 7; b.v[1] = EVP_RSQ2; break;
        case 3: b.n = 2; b.idx[0] = 2; b.v[0] = EVP_RSQ2; b.idx[1] = 6; b.v[1] = EVP_RSQ2; break;
        case 4: b.n = 2; b.idx[0] = 1; b.v[0] = EVP_RSQ2; b.idx[1] = 3; b.v[1] = EVP_RSQ2; break;
        default: b.n = 3; b.idx[0] = 0; b.v[0] = EVP_RSQ3; b.idx[1] = 4; b.v[1] = EVP_RSQ3; b.idx[2] = 8; b.v[2] = EVP_RSQ3; break;
    }
    return b;
}
// CHG_BASIS iopt=4: 3x3x3x3 -> 6x6
EVP_HD void t4_to_b66(const double* c4, double* ce) {
#pragma unroll
    for (int n = 0; n < 6; n++) {
        BasisNZ bn = basis_nz(n);
#pragma unroll
        for (int m = 0; m < 6; m++) {
            BasisNZ bm = basis_nz(m);
            double s = 0.0;
            for (int p = 0; p < bn.n; p++)
                for (int q = 0; q < bm.n; q++) s += bn.v[p] * bm.v[q] * c4[bn.idx[p] * 9 + bm.idx[q]];
            ce[n * 6 + m] = s;
        }
    }
}
// CHG_BASIS iopt=3: 6x6 -> 3x3x3x3
EVP_HD void b66_to_t4(const double* ce, double* c4) {
    for (int i = 0; i < 81; i++) c4[i] = 0.0;
    for (int n = 0; n < 6; n++) {
        BasisNZ bn = basis_nz(n);
        for (int m = 0; m < 6; m++) {
            BasisNZ bm = basis_nz(m);
            double cnm = ce[n * 6 + m];
            for (int p = 0; p < bn.n; p++)
                for (int q = 0; q < bm.n; q++) c4[bn.idx[p] * 9 + bm.idx[q]] += cnm * bn.v[p] * bm.v[q];
        }
    }
}

// VOIGT_VPSC index map (11,22,33,23,13,12) as flat 3x3 indices
EVP_HD int ijv_a(int i) { const int a[6] = {0, 1, 2, 1, 0, 0}; return a[i]; }
EVP_HD int ijv_b(int i) { const int b[6] = {0, 1, 2, 2, 2, 1}; return b[i]; }

// ---- 3x3 helpers
EVP_HD void mm3(const double* a, const double* b, double* c) {
    double t[9];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) t[3 * i + j] = a[3 * i] * b[j] + a[3 * i + 1] * b[3 + j] + a[3 * i + 2] * b[6 + j];
    for (int i = 0; i < 9; i++) c[i] = t[i];
}
EVP_HD void mm3_bt(const double* a, const double* b, double* c) {  // a * b^T
    double t[9];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) t[3 * i + j] = a[3 * i] * b[3 * j] + a[3 * i + 1] * b[3 * j + 1] + a[3 * i + 2] * b[3 * j + 2];
    for (int i = 0; i < 9; i++) c[i] = t[i];
}
EVP_HD void sym33(const double* a, double* s) {
    s[0] = a[0]; s[4] = a[4]; s[8] = a[8];
    s[1] = s[3] = 0.5 * (a[1] + a[3]);
    s[2] = s[6] = 0.5 * (a[2] + a[6]);
    s[5] = s[7] = 0.5 * (a[5] + a[7]);
}
EVP_HD void antisym33(const double* a, double* s) {
    s[0] = s[4] = s[8] = 0.0;
    s[1] = 0.5 * (a[1] - a[3]); s[2] = 0.5 * (a[2] - a[6]); s[5] = 0.5 * (a[5] - a[7]);
    s[3] = -s[1]; s[6] = -s[2]; s[7] = -s[5];
}
// determinant33 (tensor_functions.f90:442-456)
EVP_HD double det33(const double* m) {
    return m[0] * m[4] * m[8] + m[1] * m[5] * m[6] + m[2] * m[3] * m[7] - m[6] * m[4] * m[2] - m[7] * m[5] * m[0] -
           m[8] * m[3] * m[1];
}
// determinant33 of types.f90:751-756
EVP_HD double det33_cof(const double* a) {
    return a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) + a[2] * (a[3] * a[7] - a[4] * a[6]);
}
EVP_HD double frob3(const double* a) {
    double s = 0.0;
    for (int i = 0; i < 9; i++) s += a[i] * a[i];
    return sqrt(s);
}
// vm_stress / vm_strain (tensor_functions.f90:266-289)
EVP_HD double vm_stress(const double* d) {
    double h = (d[0] + d[4] + d[8]) / 3.0;
    return sqrt(3.0 / 2.0 * ((d[0] - h) * (d[0] - h) + (d[4] - h) * (d[4] - h) + (d[8] - h) * (d[8] - h) + d[1] * d[1] +
                             d[2] * d[2] + d[5] * d[5] + d[3] * d[3] + d[6] * d[6] + d[7] * d[7]));
}
EVP_HD double vm_strain(const double* d) {
    double h = (d[0] + d[4] + d[8]) / 3.0;
    return sqrt(2.0 / 3.0 * ((d[0] - h) * (d[0] - h) + (d[4] - h) * (d[4] - h) + (d[8] - h) * (d[8] - h) + d[1] * d[1] +
                             d[2] * d[2] + d[5] * d[5] + d[3] * d[3] + d[6] * d[6] + d[7] * d[7]));
}

// ---- LU with partial pivoting (dgetrf semantics: first max |a| in the column)
// In place, row-major n x n, n <= 6.  Returns 0 or k+1 for an exactly zero pivot.
EVP_HD int lu_factor(double* a, int n, int* piv) {
    int info = 0;
    for (int k = 0; k < n; k++) {
        int p = k;
        double amax = fabs(a[k * n + k]);
        for (int i = k + 1; i < n; i++) {
            double t = fabs(a[i * n + k]);
            if (t > amax) { amax = t; p = i; }
        }
        piv[k] = p;
        if (a[p * n + k] != 0.0) {
            if (p != k)
                for (int j = 0; j < n; j++) { double t = a[k * n + j]; a[k * n + j] = a[p * n + j]; a[p * n + j] = t; }
            double r = 1.0 / a[k * n + k];
            for (int i = k + 1; i < n; i++) a[i * n + k] *= r;
        } else if (info == 0) {
            info = k + 1;
        }
        for (int i = k + 1; i < n; i++) {
            double l = a[i * n + k];
            for (int j = k + 1; j < n; j++) a[i * n + j] -= l * a[k * n + j];
        }
    }
    return info;
}
EVP_HD void lu_solve(const double* lu, int n, const int* piv, double* b) {
    for (int k = 0; k < n; k++)
        if (piv[k] != k) { double t = b[k]; b[k] = b[piv[k]]; b[piv[k]] = t; }
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
// lu_inverse (tensor_functions.f90:313-337); a <- inv(a); returns info
EVP_HD int lu_inverse(double* a, int n) {
    double lu[36];
    int piv[6];
    for (int i = 0; i < n * n; i++) lu[i] = a[i];
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
EVP_HD int inv3(const double* a, double* ai) {
    for (int i = 0; i < 9; i++) ai[i] = a[i];
    return lu_inverse(ai, 3);
}

// Register-resident LU factorisation with partial pivoting (dgetrf pivot
// choice), rows swapped in place; the permutation is not recorded (dgecon
// does not use it).  Returns the dgetrf info value.
template <int n>
EVP_HD int lu_unrolled(double* J) {
    int info = 0;
#pragma unroll
    for (int k = 0; k < n; k++) {
        int p = k;
        double amax = fabs(J[k * n + k]);
#pragma unroll
        for (int i = k + 1; i < n; i++) {
            double t = fabs(J[i * n + k]);
            if (t > amax) { amax = t; p = i; }
        }
#pragma unroll
        for (int i = k + 1; i < n; i++) {
            const bool sw = (p == i);
#pragma unroll
            for (int j = 0; j < n; j++) {
                double x = J[k * n + j], y = J[i * n + j];
                J[k * n + j] = sw ? y : x;
                J[i * n + j] = sw ? x : y;
            }
        }
        const double piv = J[k * n + k];
        if (piv == 0.0 && info == 0) info = k + 1;
        const double r = 1.0 / piv;
#pragma unroll
        for (int i = k + 1; i < n; i++) {
            const double l = J[i * n + k] * r;
            J[i * n + k] = l;
#pragma unroll
            for (int j = k + 1; j < n; j++) J[i * n + j] -= l * J[k * n + j];
        }
    }
    return info;
}

// Register-resident inverse of an n x n matrix (n = 3 or 6): LU with partial
// pivoting (dgetrf pivot choice) applied to [A | I], then back substitution.
// Every index is a compile-time constant, so nothing lives in addressable
// local memory.  Returns the dgetrf info value.
template <int n>
EVP_HD int inv_unrolled(double* a) {
    double J[n * n], B[n * n];
#pragma unroll
    for (int i = 0; i < n * n; i++) {
        J[i] = a[i];
        B[i] = (i % (n + 1) == 0) ? 1.0 : 0.0;
    }
    int info = 0;
#pragma unroll
    for (int k = 0; k < n; k++) {
        int p = k;
        double amax = fabs(J[k * n + k]);
#pragma unroll
        for (int i = k + 1; i < n; i++) {
            double t = fabs(J[i * n + k]);
            if (t > amax) { amax = t; p = i; }
        }
#pragma unroll
        for (int i = k + 1; i < n; i++) {
            const bool sw = (p == i);
#pragma unroll
            for (int j = 0; j < n; j++) {
                double x = J[k * n + j], y = J[i * n + j];
                J[k * n + j] = sw ? y : x;
                J[i * n + j] = sw ? x : y;
                double u = B[k * n + j], w = B[i * n + j];
                B[k * n + j] = sw ? w : u;
                B[i * n + j] = sw ? u : w;
            }
        }
        const double piv = J[k * n + k];
        if (piv == 0.0 && info == 0) info = k + 1;
        const double r = 1.0 / piv;
#pragma unroll
        for (int i = k + 1; i < n; i++) {
            const double l = J[i * n + k] * r;
#pragma unroll
            for (int j = k + 1; j < n; j++) J[i * n + j] -= l * J[k * n + j];
#pragma unroll
            for (int j = 0; j < n; j++) B[i * n + j] -= l * B[k * n + j];
        }
    }
#pragma unroll
    for (int i = n - 1; i >= 0; i--) {
#pragma unroll
        for (int j = 0; j < n; j++) {
            double s = B[i * n + j];
#pragma unroll
            for (int m = i + 1; m < n; m++) s -= J[i * n + m] * B[m * n + j];
            B[i * n + j] = s / J[i * n + i];
        }
    }
#pragma unroll
    for (int i = 0; i < n * n; i++) a[i] = B[i];
    return info;
}
// The factors of inv_unrolled's elimination, for inverting one column at a time (a third of
// its registers: no identity block beside the matrix).  J ends with U in its upper triangle and,
// below it, each step's multiplier numerators, moved with their rows by the later
// interchanges; piv[k] is the row swapped with row k at step k.  Returns the dgetrf info value.
template <int n>
EVP_HD int lu_unrolled(double (&J)[n * n], int (&piv)[n]) {
    int info = 0;
#pragma unroll
    for (int k = 0; k < n; k++) {
        int p = k;
        double amax = fabs(J[k * n + k]);
#pragma unroll
        for (int i = k + 1; i < n; i++) {
            double t = fabs(J[i * n + k]);
            if (t > amax) { amax = t; p = i; }
        }
        piv[k] = p;
#pragma unroll
        for (int i = k + 1; i < n; i++) {
            const bool sw = (p == i);
#pragma unroll
            for (int j = 0; j < n; j++) {
                double x = J[k * n + j], y = J[i * n + j];
                J[k * n + j] = sw ? y : x;
                J[i * n + j] = sw ? x : y;
            }
        }
        const double pv = J[k * n + k];
        if (pv == 0.0 && info == 0) info = k + 1;
        const double r = 1.0 / pv;
#pragma unroll
        for (int i = k + 1; i < n; i++) {
            const double l = J[i * n + k] * r;
#pragma unroll
            for (int j = k + 1; j < n; j++) J[i * n + j] -= l * J[k * n + j];
        }
    }
    return info;
}
// Column j of the inverse from lu_unrolled's factors: the identity column through the same row
// interchanges, the eliminations of inv_unrolled in the same order with the same multipliers
// (each row takes its updates step by step either way), then its back substitution; the bits
// equal column j of inv_unrolled's result.
template <int n>
EVP_HD void lu_inverse_column(const double (&J)[n * n], const int (&piv)[n], int j, double (&x)[n]) {
    double b[n];
#pragma unroll
    for (int i = 0; i < n; i++) b[i] = (i == j) ? 1.0 : 0.0;
#pragma unroll
    for (int k = 0; k < n; k++) {
#pragma unroll
        for (int i = k + 1; i < n; i++) {
            const bool sw = (piv[k] == i);
            const double u = b[k], w = b[i];
            b[k] = sw ? w : u;
            b[i] = sw ? u : w;
        }
    }
#pragma unroll
    for (int k = 0; k < n; k++) {
        const double r = 1.0 / J[k * n + k];
#pragma unroll
        for (int i = k + 1; i < n; i++) {
            const double l = J[i * n + k] * r;
            b[i] -= l * b[k];
        }
    }
#pragma unroll
    for (int i = n - 1; i >= 0; i--) {
        double s = b[i];
#pragma unroll
        for (int m = i + 1; m < n; m++) s -= J[i * n + m] * x[m];
        x[i] = s / J[i * n + i];
    }
}
EVP_HD int inv3u(const double* a, double* ai) {
#pragma unroll
    for (int i = 0; i < 9; i++) ai[i] = a[i];
    return inv_unrolled<3>(ai);
}

// Register-resident 6x6 solve J x = b with partial pivoting (dgesv), fully unrolled.
EVP_HD int solve6(double (&J)[36], double (&b)[6]) {
    int info = 0;
#pragma unroll
    for (int k = 0; k < 6; k++) {
        int p = k;
        double amax = fabs(J[k * 6 + k]);
#pragma unroll
        for (int i = k + 1; i < 6; i++) {
            double t = fabs(J[i * 6 + k]);
            if (t > amax) { amax = t; p = i; }
        }
#pragma unroll
        for (int i = k + 1; i < 6; i++) {
            bool sw = (p == i);
#pragma unroll
            for (int j = 0; j < 6; j++) {
                double a = J[k * 6 + j], c = J[i * 6 + j];
                J[k * 6 + j] = sw ? c : a;
                J[i * 6 + j] = sw ? a : c;
            }
            double a = b[k], c = b[i];
            b[k] = sw ? c : a;
            b[i] = sw ? a : c;
        }
        double piv = J[k * 6 + k];
        if (piv == 0.0 && info == 0) info = k + 1;
        double r = 1.0 / piv;
#pragma unroll
        for (int i = k + 1; i < 6; i++) {
            double l = J[i * 6 + k] * r;
            J[i * 6 + k] = l;
#pragma unroll
            for (int j = k + 1; j < 6; j++) J[i * 6 + j] -= l * J[k * 6 + j];
            b[i] -= l * b[k];
        }
    }
#pragma unroll
    for (int i = 5; i >= 0; i--) {
        double s = b[i];
#pragma unroll
        for (int j = i + 1; j < 6; j++) s -= J[i * 6 + j] * b[j];
        b[i] = s / J[i * 6 + i];
    }
    return info;
}

// ---- matrix exponential (various_functions.f90:1829-1967)
EVP_HD double l1_norm33(const double* m) {
    double l1 = 0.0;
    for (int j = 0; j < 3; j++) {
        double cs = fabs(m[j]) + fabs(m[3 + j]) + fabs(m[6 + j]);
        if (cs > l1) l1 = cs;
    }
    return l1;
}
EVP_HD int expm_adaptive(const double* a, double* e) {
    if (l1_norm33(a) <= 1.0e-1) {
        double a2[9], a3[9];
        mm3(a, a, a2);
        mm3(a2, a, a3);
        for (int i = 0; i < 9; i++) e[i] = ((i % 4 == 0) ? 1.0 : 0.0) + a[i] + a2[i] / 2.0 + a3[i] / 6.0;
        return 0;
    }
    const double theta13 = 5.371920351148152;
    const double b0 = 64764752532480000.0, b1 = 32382376266240000.0, b2 = 7771770303897600.0, b3 = 1187353796428800.0,
                 b4 = 129060195264000.0, b5 = 10559470521600.0, b6 = 670442572800.0, b7 = 33522128640.0, b8 = 1323241920.0,
                 b9 = 40840800.0, b10 = 960960.0, b11 = 16380.0, b12 = 182.0, b13 = 1.0;
    double A[9];
    double normA = l1_norm33(a);
    if (!(normA < 1.0e300)) {  // non-finite input: report instead of squaring without end
        for (int i = 0; i < 9; i++) e[i] = normA;
        return -1;
    }
    int s = 0;
    if (normA > theta13) s = (int)ceil(log(normA / theta13) / log(2.0));
    double sc = pow(2.0, (double)s);
    for (int i = 0; i < 9; i++) A[i] = a[i] / sc;
    double A2[9], A4[9], A6[9], t1[9], t2[9], U[9], V[9];
    mm3(A, A, A2); mm3(A2, A2, A4); mm3(A2, A4, A6);
    for (int i = 0; i < 9; i++) t1[i] = b13 * A6[i] + b11 * A4[i] + b9 * A2[i];
    mm3(A6, t1, t2);
    for (int i = 0; i < 9; i++) t2[i] = t2[i] + b7 * A6[i] + b5 * A4[i] + b3 * A2[i] + b1 * ((i % 4 == 0) ? 1.0 : 0.0);
    mm3(A, t2, U);
    for (int i = 0; i < 9; i++) t1[i] = b12 * A6[i] + b10 * A4[i] + b8 * A2[i];
    mm3(A6, t1, V);
    for (int i = 0; i < 9; i++) V[i] = V[i] + b6 * A6[i] + b4 * A4[i] + b2 * A2[i] + b0 * ((i % 4 == 0) ? 1.0 : 0.0);
    double Q[9], P[9];
    for (int i = 0; i < 9; i++) { Q[i] = V[i] - U[i]; P[i] = V[i] + U[i]; }
    int info = inv_unrolled<3>(Q);
    if (info != 0) return info;
    mm3(Q, P, e);
    for (int k = 0; k < s; k++) mm3(e, e, e);
    return 0;
}

// ---- polar decomposition F = R U (polar_dcmp, tensor_functions.f90:367-393).
// The factor is unique for det F != 0; computed by the scaled Newton iteration
// X <- (g X + X^{-T}/g)/2 (Higham 1986).
EVP_HD void adj_inv3(const double* a, double* inv) {
    double c00 = a[4] * a[8] - a[5] * a[7];
    double c01 = a[5] * a[6] - a[3] * a[8];
    double c02 = a[3] * a[7] - a[4] * a[6];
    double det = a[0] * c00 + a[1] * c01 + a[2] * c02;
    double r = 1.0 / det;
    inv[0] = c00 * r; inv[3] = c01 * r; inv[6] = c02 * r;
    inv[1] = (a[2] * a[7] - a[1] * a[8]) * r;
    inv[4] = (a[0] * a[8] - a[2] * a[6]) * r;
    inv[7] = (a[1] * a[6] - a[0] * a[7]) * r;
    inv[2] = (a[1] * a[5] - a[2] * a[4]) * r;
    inv[5] = (a[2] * a[3] - a[0] * a[5]) * r;
    inv[8] = (a[0] * a[4] - a[1] * a[3]) * r;
}
EVP_HD void polar(const double* F, double* R, double* U) {
    double X[9], Xi[9];
    for (int i = 0; i < 9; i++) X[i] = F[i];
    bool scale = true;
    for (int it = 0; it < 60; it++) {
        adj_inv3(X, Xi);
        double g = 1.0;
        if (scale) g = sqrt(frob3(Xi) / frob3(X));
        double d = 0.0, nn = 0.0;
        double Xn[9];
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) {
                Xn[3 * i + j] = 0.5 * (g * X[3 * i + j] + Xi[3 * j + i] / g);
                double df = Xn[3 * i + j] - X[3 * i + j];
                d += df * df;
                nn += Xn[3 * i + j] * Xn[3 * i + j];
            }
        for (int i = 0; i < 9; i++) X[i] = Xn[i];
        if (d <= 1e-20 * nn) scale = false;
        if (d <= 1e-30 * nn) break;
    }
    for (int i = 0; i < 9; i++) R[i] = X[i];
    double Ut[9];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) Ut[3 * i + j] = R[i] * F[j] + R[3 + i] * F[3 + j] + R[6 + i] * F[6 + j];  // R^T F
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) U[3 * i + j] = 0.5 * (Ut[3 * i + j] + Ut[3 * j + i]);
}

// ---- symmetric 3x3 eigen-decomposition (dsyev 'V','U'): cyclic Jacobi, ascending.
EVP_HD void sym_eig3(const double* A, double* w, double* Q) {
    double a[9];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) a[3 * i + j] = (i <= j) ? A[3 * i + j] : A[3 * j + i];
    for (int i = 0; i < 9; i++) Q[i] = (i % 4 == 0) ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 60; sweep++) {
        double off = a[1] * a[1] + a[2] * a[2] + a[5] * a[5];
        if (off == 0.0) break;
        double diag = a[0] * a[0] + a[4] * a[4] + a[8] * a[8];
        if (off < 1e-36 * diag) break;
        for (int p = 0; p < 2; p++)
            for (int q = p + 1; q < 3; q++) {
                double apq = a[3 * p + q];
                if (apq == 0.0) continue;
                double theta = (a[3 * q + q] - a[3 * p + p]) / (2.0 * apq);
                double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < 3; k++) {
                    double akp = a[3 * k + p], akq = a[3 * k + q];
                    a[3 * k + p] = c * akp - s * akq;
                    a[3 * k + q] = s * akp + c * akq;
                }
                for (int k = 0; k < 3; k++) {
                    double apk = a[3 * p + k], aqk = a[3 * q + k];
                    a[3 * p + k] = c * apk - s * aqk;
                    a[3 * q + k] = s * apk + c * aqk;
                }
                for (int k = 0; k < 3; k++) {
                    double qkp = Q[3 * k + p], qkq = Q[3 * k + q];
                    Q[3 * k + p] = c * qkp - s * qkq;
                    Q[3 * k + q] = s * qkp + c * qkq;
                }
            }
    }
    double d[3] = {a[0], a[4], a[8]};
    int i0 = 0, i1 = 1, i2 = 2, t;
    if (d[i1] < d[i0]) { t = i0; i0 = i1; i1 = t; }
    if (d[i2] < d[i1]) { t = i1; i1 = i2; i2 = t; }
    if (d[i1] < d[i0]) { t = i0; i0 = i1; i1 = t; }
    int idx[3] = {i0, i1, i2};
    double Qs[9];
    for (int c = 0; c < 3; c++) {
        w[c] = d[idx[c]];
        for (int r = 0; r < 3; r++) Qs[3 * r + c] = Q[3 * r + idx[c]];
    }
    for (int i = 0; i < 9; i++) Q[i] = Qs[i];
}

// Incremental kinematics of kinematic_increments / update_diagnostics:
// |log J|, rotation angle (deg) of the polar rotation, ||log U||_F.
EVP_HD void stretch_rot(const double* Finc, bool cof_det, double& volinc, double& rotang, double& stretchinc, double& Jinc) {
    Jinc = cof_det ? det33_cof(Finc) : det33(Finc);
    volinc = fabs(log(fmax(Jinc, EVP_TINY)));
    double R[9], U[9];
    polar(Finc, R, U);
    double arg = 0.5 * ((R[0] + R[4] + R[8]) - 1.0);
    arg = fmax(-1.0, fmin(1.0, arg));
    rotang = acos(arg) * 180 / EVP_PI;
    double w[3], Q[9], tm[9], lu[9];
    sym_eig3(U, w, Q);
    for (int ii = 0; ii < 3; ii++) {
        double lw = log(fmax(w[ii], EVP_TINY));
        for (int r = 0; r < 3; r++) tm[3 * r + ii] = Q[3 * r + ii] * lw;
    }
    mm3_bt(tm, Q, lu);
    stretchinc = frob3(lu);
}

// ---- 1-norm condition estimate (dgetrf + dgecon): Hager/Higham estimator
// (Higham 1988, Algorithm 4.1) on the LU factors without the row permutation.
EVP_HD double cond1_est_6x6(const double* Ain) {
    const int n = 6;
    double lu[36];
    double anorm = 0.0;
    for (int j = 0; j < n; j++) {
        double cs = 0.0;
        for (int i = 0; i < n; i++) cs += fabs(Ain[i * n + j]);
        anorm = fmax(anorm, cs);
    }
    for (int i = 0; i < 36; i++) lu[i] = Ain[i];
    if (lu_unrolled<6>(lu) != 0) return EVP_HUGE;
    double x[6], v[6];
    int isgn[6];
    auto solveA = [&](double* y) {
        for (int i = 0; i < n; i++) { double s = y[i]; for (int j = 0; j < i; j++) s -= lu[i * n + j] * y[j]; y[i] = s; }
        for (int i = n - 1; i >= 0; i--) { double s = y[i]; for (int j = i + 1; j < n; j++) s -= lu[i * n + j] * y[j]; y[i] = s / lu[i * n + i]; }
    };
    auto solveAT = [&](double* y) {
        for (int i = 0; i < n; i++) { double s = y[i]; for (int j = 0; j < i; j++) s -= lu[j * n + i] * y[j]; y[i] = s / lu[i * n + i]; }
        for (int i = n - 1; i >= 0; i--) { double s = y[i]; for (int j = i + 1; j < n; j++) s -= lu[j * n + i] * y[j]; y[i] = s; }
    };
    auto dasum = [&](const double* y) { double s = 0; for (int i = 0; i < n; i++) s += fabs(y[i]); return s; };
    auto idamax = [&](const double* y) { int k = 0; double m = fabs(y[0]); for (int i = 1; i < n; i++) if (fabs(y[i]) > m) { m = fabs(y[i]); k = i; } return k; };
    for (int i = 0; i < n; i++) x[i] = 1.0 / n;
    solveA(x);
    double est = dasum(x);
    for (int i = 0; i < n; i++) { x[i] = (x[i] >= 0.0) ? 1.0 : -1.0; isgn[i] = (x[i] > 0.0) ? 1 : -1; }
    solveAT(x);
    int j = idamax(x);
    int iter = 2;
    for (int guard = 0; guard < 8; guard++) {
        for (int i = 0; i < n; i++) x[i] = 0.0;
        x[j] = 1.0;
        solveA(x);
        for (int i = 0; i < n; i++) v[i] = x[i];
        double estold = est;
        est = dasum(v);
        bool changed = false;
        for (int i = 0; i < n; i++) {
            int xs = (x[i] >= 0.0) ? 1 : -1;
            if (xs != isgn[i]) { changed = true; break; }
        }
        if (!changed) break;
        if (est <= estold) break;
        for (int i = 0; i < n; i++) { x[i] = (x[i] >= 0.0) ? 1.0 : -1.0; isgn[i] = (x[i] > 0.0) ? 1 : -1; }
        solveAT(x);
        int jlast = j;
        j = idamax(x);
        if ((x[jlast] != fabs(x[j])) && (iter < 5)) { iter++; continue; }
        break;
    }
    double altsgn = 1.0;
    for (int i = 0; i < n; i++) { x[i] = altsgn * (1.0 + (double)i / (double)(n - 1)); altsgn = -altsgn; }
    solveA(x);
    double temp = 2.0 * (dasum(x) / (double)(3 * n));
    if (temp > est) est = temp;
    if (est == 0.0) return EVP_HUGE;
    double rcond = (1.0 / est) / anorm;
    if (!(rcond > 0.0)) return EVP_HUGE;
    return 1.0 / rcond;
}

// rotate a 4th-order tensor: out_ijkl = A_iI A_jJ A_kK A_lL in_IJKL (one index at a time)
EVP_HD void rotate4(const double* A, const double* in, double* out) {
    double t1[81], t2[81];
    for (int i = 0; i < 3; i++) for (int r = 0; r < 27; r++) {
        double s = 0; for (int I = 0; I < 3; I++) s += A[3 * i + I] * in[I * 27 + r]; t1[i * 27 + r] = s; }
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) for (int r = 0; r < 9; r++) {
        double s = 0; for (int J = 0; J < 3; J++) s += A[3 * j + J] * t1[i * 27 + J * 9 + r]; t2[i * 27 + j * 9 + r] = s; }
    for (int ij = 0; ij < 9; ij++) for (int k = 0; k < 3; k++) for (int L = 0; L < 3; L++) {
        double s = 0; for (int K = 0; K < 3; K++) s += A[3 * k + K] * t2[ij * 9 + K * 3 + L]; t1[ij * 9 + k * 3 + L] = s; }
    for (int ijk = 0; ijk < 27; ijk++) for (int l = 0; l < 3; l++) {
        double s = 0; for (int L = 0; L < 3; L++) s += A[3 * l + L] * t1[ijk * 3 + L]; out[ijk * 3 + l] = s; }
}

// The b-basis form of the rotation c'_ijkl = a_ip a_jq a_kr a_ls c_pqrs of a fourth-order tensor
// with minor symmetries: c'66 = Q c66 Q^T with Q_ag = <B^a, a B^g a^T> (Frobenius product; B^0..B^5
// the symmetric basis of chg_basis, complete for symmetric 3x3 tensors).  Q[6 * a + g].
EVP_HD void rot_b66(const double* a, double* Q) {
#pragma unroll
    for (int g = 0; g < 6; g++) {
        const BasisNZ bg = basis_nz(g);
        double Bg[9], t[9], M[9];
#pragma unroll
        for (int c = 0; c < 9; c++) Bg[c] = 0.0;
#pragma unroll
        for (int p = 0; p < 3; p++)
            if (p < bg.n) Bg[bg.idx[p]] = bg.v[p];
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) {
                double s = 0.0;
#pragma unroll
                for (int k = 0; k < 3; k++) s += a[3 * i + k] * Bg[3 * k + j];
                t[3 * i + j] = s;
            }
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) {
                double s = 0.0;
#pragma unroll
                for (int k = 0; k < 3; k++) s += t[3 * i + k] * a[3 * j + k];
                M[3 * i + j] = s;
            }
#pragma unroll
        for (int al = 0; al < 6; al++) {
            const BasisNZ ba = basis_nz(al);
            double s = 0.0;
#pragma unroll
            for (int p = 0; p < 3; p++)
                if (p < ba.n) s += ba.v[p] * M[ba.idx[p]];
            Q[6 * al + g] = s;
        }
    }
}

// euler(iopt=2) (tensor_functions.f90:550-566)
EVP_HD void euler2(double ph, double th, double tm, double* a) {
    double sph = sin(ph), cph = cos(ph), sth = sin(th), cth = cos(th), stm = sin(tm), ctm = cos(tm);
    a[0] = ctm * cph - sph * stm * cth;
    a[3] = -stm * cph - sph * ctm * cth;
    a[6] = sph * sth;
    a[1] = ctm * sph + cph * stm * cth;
    a[4] = -sph * stm + cph * ctm * cth;
    a[7] = -sth * cph;
    a[2] = sth * stm;
    a[5] = ctm * sth;
    a[8] = cth;
}

}  // namespace evp
