// evp_kernels.cu -- per-voxel sm_100a kernels of the LS-EVPFFT solve.
//
// One thread per voxel (grid-stride), SoA FP64 state (layout in evp_dev.cuh).
// Every reduction is a fixed-order tree: warp shuffles, one partial per block,
// and the last block to finish sums the partials in block order, so results
// are reproducible run to run.  Kernel <-> reference routine map:
//   k_init      data_grain + Hall-Petch init + initial_guess (IO_functions.f90:722-812, 107-199;
//               various_functions.f90:8-53) and the start-up c066 sum (LS-EVPFFT.f90:156-165)
//   k_sgavg     stress average before the PK1 prologue (LS-EVPFFT.f90:238-254)
//   k_prologue  update_schmid + calc_c066mod_Goperr066mod (various_functions.f90:472-539, 812-906)
//   k_gas_compl calc_gas_compl (various_functions.f90:909-951)
//   k_corr      correction_to_current pass 2 + velgrad mixing (various_functions.f90:1103-1139;
//               LS-EVPFFT.f90:277-311)
//   k_newton    solve_res / plastic_strain_rate / elastic_strain_rate / harden
//               (various_functions.f90:1142-1491) + the stress sums of calc_velgradavg_corr (1556-1578)
//   k_upd1      accepted-step commit (LS-EVPFFT.f90:432-446) + update_plastic_defgrad + update_defgrad
//   k_upd2      update_elstic_defgrad + update_el_stiff + update_tensor_config pass 1
//   k_upd3      update_tensor_config pass 2 + update_hardening + macro averages (LS-EVPFFT.f90:460-523)
//   k_diag      update_diagnostics (types.f90:345-692)
//   k_c0        calc_c0 voxel part (various_functions.f90:2537-2634)
//   k_kinematic kinematic_increments (various_functions.f90:2766-2837)
//   k_goperr0   real-space Green operator at the origin (various_functions.f90:798-807)
//   k_cell2node cell2node_tensor1 + nodal update (various_functions.f90:2026-2054, 2652-2691)
#include "evp_dev.cuh"
#include "evp_math.cuh"

#include <cstdio>
#include <cstdlib>
#include <mutex>

namespace evp {

constexpr int kBlock = 256;
constexpr int kNewtonBlock = 128;
constexpr int kC0Block = 64;

// ---------------------------------------------------------------- reductions
// NS sums then NM maxima per thread -> one partial per block (stored field-major,
// partials[f * nblocks + block], in the body's block coordinates) -> the last block to finish folds them: one
// warp per field, lane l adding blocks l, l + 32, ... in order, then a fixed
// shuffle tree, so the result does not depend on timing (fold_sum, in evp_dev.cuh, for the
// sums; fold_max for the maxima).
__device__ __forceinline__ double fold_max(const double* partials, int nblk, int f, int lane) {
    const double* q = partials + (size_t)f * nblk;
    double s = -EVP_HUGE;
    int b = lane;
    for (; b + 7 * 32 < nblk; b += 8 * 32) {
        double x[8];
#pragma unroll
        for (int i = 0; i < 8; i++) x[i] = __ldcg(q + b + 32 * i);
#pragma unroll
        for (int i = 0; i < 8; i++) s = fmax(s, x[i]);
    }
    for (; b < nblk; b += 32) s = fmax(s, __ldcg(q + b));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s = fmax(s, __shfl_down_sync(0xffffffffu, s, o));
    return s;  // in lane 0
}

template <int NS, int NM>
__device__ void reduce_store(const double* sums, const double* maxs, double* partials, double* out, unsigned int* counter,
                             const VB& vb) {
    constexpr int NF = NS + NM;
    __shared__ double sh[NF][32];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int f = 0; f < NF; f++) {
        double x = (f < NS) ? sums[f] : maxs[f - NS];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            double y = __shfl_down_sync(0xffffffffu, x, o);
            x = (f < NS) ? x + y : fmax(x, y);
        }
        if (lane == 0) sh[f][warp] = x;
    }
    __syncthreads();
    if (warp == 0) {
        for (int f = 0; f < NF; f++) {
            double x = (lane < nw) ? sh[f][lane] : ((f < NS) ? 0.0 : -EVP_HUGE);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                double y = __shfl_down_sync(0xffffffffu, x, o);
                x = (f < NS) ? x + y : fmax(x, y);
            }
            if (lane == 0) partials[(size_t)f * vb.nx + vb.x] = x;
        }
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = (atomicAdd(counter, 1u) == (unsigned)vb.nx - 1u);
    __syncthreads();
    if (last) {
        __threadfence();
        for (int f = warp; f < NF; f += nw) {
            const double x = (f < NS) ? fold_sum(partials, vb.nx, f, lane) : fold_max(partials, vb.nx, f, lane);
            if (lane == 0) out[f] = x;
        }
        if (threadIdx.x == 0) *counter = 0;
    }
}

__device__ __forceinline__ void set_err(int* err, int bit) { atomicOr(err, bit); }

__device__ __forceinline__ void ld9(const double* __restrict__ a, long long N, long long v, double* o) {
#pragma unroll
    for (int c = 0; c < 9; c++) o[c] = a[c * N + v];
}
__device__ __forceinline__ void st9(double* __restrict__ a, long long N, long long v, const double* o) {
#pragma unroll
    for (int c = 0; c < 9; c++) a[c * N + v] = o[c];
}
__device__ __forceinline__ void ld6(const double* __restrict__ a, long long N, long long v, double* o) {
#pragma unroll
    for (int c = 0; c < 6; c++) o[c] = a[c * N + v];
}
__device__ __forceinline__ void st6(double* __restrict__ a, long long N, long long v, const double* o) {
#pragma unroll
    for (int c = 0; c < 6; c++) a[c * N + v] = o[c];
}
__device__ __forceinline__ void eye9(double* a) {
#pragma unroll
    for (int c = 0; c < 9; c++) a[c] = (c % 4 == 0) ? 1.0 : 0.0;
}

// |x|^e for the power law: integer exponents by binary powering, else pow().
__device__ __forceinline__ double powabs(double x, double e, int int_exp) {
    double a = fabs(x);
    if (int_exp) {
        int k = (int)e;
        double r = 1.0, b = a;
        while (k) {
            if (k & 1) r *= b;
            b *= b;
            k >>= 1;
        }
        return r;
    }
    return pow(a, e);
}

// ---------------------------------------------------------------- k_init
struct InitParams {
    double udot[9];
    double u6t[6];  // b6(udot) * tdot of process 1
    int keepF;       // F, F^-1, det F and w J come from k_dispini
    double detFavg;  // sum of w J (divides the weights when keepF)
};

__global__ void __launch_bounds__(kBlock) k_init(Dev d, const double* __restrict__ euler, const int* __restrict__ grain,
                                                   const double* __restrict__ hp, InitParams ip) {
    const long long N = d.N;
    double sums[36];
#pragma unroll
    for (int c = 0; c < 36; c++) sums[c] = 0.0;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < N; v += (long long)gridDim.x * blockDim.x) {
        const int p = d.phase[v];
        const PhaseDev& ph = d.ph[p];
        double I9[9];
        eye9(I9);
        if (!ip.keepF) {
            st9(d.F, N, v, I9);
            st9(d.Finv, N, v, I9);
            d.detF[v] = 1.0;
        }
        st9(d.Fe, N, v, I9); st9(d.Fp, N, v, I9);
        st9(d.Finc, N, v, I9); st9(d.Feinc, N, v, I9);
        const double w = ip.keepF ? d.wgtc[v] / ip.detFavg : d.wgt;  // wgtc (IO_functions.f90:917, 934)
        d.wgtc[v] = w;
        d.epvm[v] = 0.0;
        d.gacumgr[v] = 0.0;
        st9(d.velgrad, N, v, ip.udot);
        double z[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        st9(d.velgradold, N, v, z);
        st9(d.dvr, N, v, z);
        st6(d.sgt, N, v, z); st6(d.edotp, N, v, z); st6(d.ept, N, v, z); st6(d.disgradsym, N, v, z);
        for (int s = 0; s < d.nsys; s++) {
            d.gamdot[s * N + v] = 0.0;
            d.crss[(2 * s) * N + v] = 0.0; d.crss[(2 * s + 1) * N + v] = 0.0;
            d.trialtau[(2 * s) * N + v] = 0.0; d.trialtau[(2 * s + 1) * N + v] = 0.0;
            for (int c = 0; c < 5; c++) d.sch[(s * 5 + c) * N + v] = 0.0;
        }
        if (ph.igas) {
            st6(d.sg, N, v, z);
            st9(d.ag, N, v, z);
            for (int c = 0; c < 36; c++) d.sg66[c * N + v] = 0.0;
            continue;
        }
        double aa[9], ag[9];
        const double deg = EVP_PI / 180.0;
        euler2(euler[3 * v] * deg, euler[3 * v + 1] * deg, euler[3 * v + 2] * deg, aa);
        for (int j = 0; j < 3; j++)
            for (int k = 0; k < 3; k++) ag[3 * j + k] = aa[3 * k + j];
        st9(d.ag, N, v, ag);
        double c4[81], cg66[36];
        rotate4(ag, ph.C, c4);
        t4_to_b66(c4, cg66);
        for (int c = 0; c < 36; c++) sums[c] += cg66[c] * w;
        double sg6[6], s6[6];
        for (int i = 0; i < 6; i++) {
            double s = 0.0;
            for (int j = 0; j < 6; j++) s += cg66[6 * i + j] * ip.u6t[j];
            sg6[i] = s;
        }
        b6_to_s6(sg6, s6);
        st6(d.sg, N, v, s6);
        if (inv_unrolled<6>(cg66) != 0) set_err(d.err, 1);
        for (int c = 0; c < 36; c++) d.sg66[c * N + v] = cg66[c];
        const double hps = hp[v];
        for (int s = 0; s < ph.nsyst; s++) {
            double c1 = ph.tau0f[s] + hps, c2 = ph.tau0b[s] + hps;
            double db1 = ag[3] * ph.dbca[3 * s] + ag[4] * ph.dbca[3 * s + 1] + ag[5] * ph.dbca[3 * s + 2];
            double cosalpha = fabs(db1);
            c1 = c1 + ph.hpfac[s] * sqrt(cosalpha);
            c2 = c2 + ph.hpfac[s] * sqrt(cosalpha);
            d.crss[(2 * s) * N + v] = c1;
            d.crss[(2 * s + 1) * N + v] = c2;
            d.trialtau[(2 * s) * N + v] = c2;  // both columns start from the backward CRSS (IO_functions.f90:193-194)
            d.trialtau[(2 * s + 1) * N + v] = c2;
        }
    }
    reduce_store<36, 0>(sums, nullptr, d.partials, d.red + OFF_INIT, d.counters + CNT_INIT, hw_vb());
}

void launch_init(const Dev& d, const double* euler, const int* grain, const double* hp, const double* udot9, const double* u6t,
                 int keepF, double detFavg, cudaStream_t st) {
    InitParams ip;
    for (int c = 0; c < 9; c++) ip.udot[c] = udot9[c];
    for (int c = 0; c < 6; c++) ip.u6t[c] = u6t[c];
    ip.keepF = keepF;
    ip.detFavg = detFavg;
    k_init<<<d.grid, kBlock, 0, st>>>(d, euler, grain, hp, ip);
}

// ---------------------------------------------------------------- k_dispini
// init_defgrad per voxel (IO_functions.f90:893-921).  Sums, in OFF_DISP order: F^-1 w J over all
// voxels (9), the solid ones (9), the gas ones (9); w J over solid and gas voxels; J w.
__global__ void __launch_bounds__(kBlock) k_dispini(Dev d, const double* __restrict__ grad, double delt) {
    const long long N = d.N;
    double sums[30];
#pragma unroll
    for (int c = 0; c < 30; c++) sums[c] = 0.0;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < N; v += (long long)gridDim.x * blockDim.x) {
        double F[9], Fi[9];
        for (int l = 0; l < 3; l++)
            for (int m = 0; m < 3; m++) F[3 * l + m] = grad[(size_t)(3 * m + l) * N + v] + (l == m ? delt : 0.0);
        const double J = det33(F);
        if (inv3u(F, Fi) != 0) set_err(d.err, 1);
        st9(d.F, N, v, F);
        st9(d.Fini, N, v, F);
        st9(d.Finv, N, v, Fi);
        d.detF[v] = J;
        d.wgtc[v] = d.wgt * J;
        const int gas = d.gas[v];
#pragma unroll
        for (int c = 0; c < 9; c++) {
            const double t = Fi[c] * d.wgt * J;
            sums[c] += t;
            sums[9 + c] += gas ? 0.0 : t;
            sums[18 + c] += gas ? t : 0.0;
        }
        sums[27] += gas ? 0.0 : d.wgt * J;
        sums[28] += gas ? d.wgt * J : 0.0;
        sums[29] += J * d.wgt;
    }
    reduce_store<30, 0>(sums, nullptr, d.partials, d.red + OFF_DISP, d.counters + CNT_DISP, hw_vb());
}
void launch_dispini(const Dev& d, const double* grad, double delt, cudaStream_t st) {
    k_dispini<<<d.grid, kBlock, 0, st>>>(d, grad, delt);
}

// ---------------------------------------------------------------- k_sgavg
__device__ __forceinline__ void body_sgavg(const Dev& d, const VB& vb) {
    const long long N = d.N;
    double s[6] = {0, 0, 0, 0, 0, 0};
    for (long long v = vb.x * (long long)blockDim.x + threadIdx.x; v < N; v += (long long)vb.nx * blockDim.x) {
        double w = d.wgtc[v];
#pragma unroll
        for (int c = 0; c < 6; c++) s[c] += d.sg[c * N + v] * w;
    }
    reduce_store<6, 0>(s, nullptr, d.partials, d.red + OFF_SGAVG, d.counters + CNT_SGAVG, vb);
}
__global__ void __launch_bounds__(kBlock) k_sgavg(Dev d) { body_sgavg(d, hw_vb()); }
void launch_sgavg(const Dev& d, cudaStream_t st) { k_sgavg<<<d.grid, kBlock, 0, st>>>(d); }

// ---------------------------------------------------------------- b-basis congruence
// For a 3x3 matrix M, T(M)_ag = <B^a, B^g M^T> (Frobenius product; B^0..B^5 the orthonormal
// b-basis of chg_basis).  A fourth-order tensor with minor symmetries, c = sum B^g c66_gd B^d,
// pulled back as p_ijkl = sum_mn c_imkn M_jm M_ln has the b-basis components T c66 T^T, so the
// 3x3x3x3 expansion and its contraction (81 x 9 products) reduce to two 6x6 products.
__device__ __forceinline__ void basis_T(const double* M, double* T) {
    double Bg[9], P[9], col[6];
#pragma unroll
    for (int g = 0; g < 6; g++) {
#pragma unroll
        for (int c = 0; c < 9; c++) Bg[c] = 0.0;
        if (g == 0) { Bg[0] = -EVP_RSQ2; Bg[4] = EVP_RSQ2; }
        else if (g == 1) { Bg[0] = -EVP_RSQ6; Bg[4] = -EVP_RSQ6; Bg[8] = EVP_RSQ23; }
        else if (g == 2) { Bg[5] = EVP_RSQ2; Bg[7] = EVP_RSQ2; }
        else if (g == 3) { Bg[2] = EVP_RSQ2; Bg[6] = EVP_RSQ2; }
        else if (g == 4) { Bg[1] = EVP_RSQ2; Bg[3] = EVP_RSQ2; }
        else { Bg[0] = EVP_RSQ3; Bg[4] = EVP_RSQ3; Bg[8] = EVP_RSQ3; }
        mm3_bt(Bg, M, P);  // B^g M^T
        t2_to_b6(P, col);
#pragma unroll
        for (int a = 0; a < 6; a++) T[6 * a + g] = col[a];
    }
}
// out = s * T A T^T (6x6)
// (a row of T A at a time: six live values instead of 36, each sum in the same order)
__device__ __forceinline__ void congruence6(const double* T, const double* A, double s, double* out) {
#pragma unroll
    for (int i = 0; i < 6; i++) {
        double ta[6];
#pragma unroll
        for (int j = 0; j < 6; j++) {
            double x = 0.0;
#pragma unroll
            for (int k = 0; k < 6; k++) x += T[6 * i + k] * A[6 * k + j];
            ta[j] = x;
        }
#pragma unroll
        for (int j = 0; j < 6; j++) {
            double x = 0.0;
#pragma unroll
            for (int k = 0; k < 6; k++) x += ta[k] * T[6 * j + k];
            out[6 * i + j] = s * x;
        }
    }
}

// ---------------------------------------------------------------- k_prologue
// One block of 256 per SM at most (200 registers): the C~ congruence and its LU factors stay in
// registers, where a two-block bound of 128 registers spilled ~0.5 kB per thread to local memory
// (its write-back nearly doubled the kernel's DRAM writes).
__global__ void __launch_bounds__(kBlock, 1) k_prologue(Dev d, const double* __restrict__ c0g, const double* __restrict__ g0g,
                                                       int do_schmid, int modal) {
    __shared__ double c0[81], g0[81], c0b[36];
    for (int i = threadIdx.x; i < 81; i += blockDim.x) {
        c0[i] = c0g[i];
        g0[i] = modal ? g0g[i] : 0.0;
    }
    __syncthreads();
    if (threadIdx.x == 0) t4_to_b66(c0, c0b);
    __syncthreads();
    const long long N = d.N;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < N; v += (long long)gridDim.x * blockDim.x) {
        const bool gas = d.gas[v];
        if (do_schmid && !gas) {
            const PhaseDev& ph = d.ph[d.phase[v]];
            double Fe[9], ag[9], aa[9], ai[9];
            ld9(d.Fe, N, v, Fe);
            ld9(d.ag, N, v, ag);
            mm3(Fe, ag, aa);
            if (inv3u(aa, ai) != 0) set_err(d.err, 1);
            for (int s = 0; s < ph.nsyst; s++) {
                double S[9], t[9], r[9], rs[9], b5[5];
#pragma unroll
                for (int i = 0; i < 3; i++)
#pragma unroll
                    for (int j = 0; j < 3; j++) S[3 * i + j] = ph.dbca[3 * s + i] * ph.dnca[3 * s + j];
                mm3(aa, S, t);
                mm3(t, ai, r);
                sym33(r, rs);
                t2_to_b5(rs, b5);
#pragma unroll
                for (int c = 0; c < 5; c++) d.sch[(s * 5 + c) * N + v] = b5[c];
            }
        }
        double F[9], detF = d.detF[v];
        ld9(d.F, N, v, F);
        // calc_c066mod: cm_ijkl = sum_mn c0_imkn F_jm F_ln / J, quarter-symmetrized, in the b-basis;
        // c0 has the minor symmetries, so this is (1/J) T(F) c0_66 T(F)^T
        double c66[36], TF[36];
        basis_T(F, TF);
        congruence6(TF, c0b, 1.0 / detF, c66);
#pragma unroll
        for (int c = 0; c < 36; c++) d.c066mod[c * N + v] = c66[c];
        // its inverse, for the symmetric form of the local Newton system, a column at a time from
        // the LU factors (the bits of inv_unrolled without its identity block in registers)
        int piv[6];
        if (lu_unrolled<6>(c66, piv) != 0 && !gas) set_err(d.err, 1);
#pragma unroll
        for (int j = 0; j < 6; j++) {
            double x[6];
            lu_inverse_column<6>(c66, piv, j, x);
#pragma unroll
            for (int i = 0; i < 6; i++) d.c066inv[(6 * i + j) * N + v] = x[i];
        }
    }
}
// calc_c066mod_Goperr066mod, the modified augmented Lagrangian part (various_functions.f90:866-900):
// cG = C~ : Gamma~r with Gamma~r = sym(J Gamma^r(0) F^-1 F^-1), for --modal 1 only (a kernel of its
// own, so that its 3x3x3x3 work arrays do not burden the common prologue's registers)
__global__ void __launch_bounds__(kBlock, 2) k_prologue_modal(Dev d, const double* __restrict__ g0g) {
    __shared__ double g0[81];
    for (int i = threadIdx.x; i < 81; i += blockDim.x) g0[i] = g0g[i];
    __syncthreads();
    const long long N = d.N;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < N; v += (long long)gridDim.x * blockDim.x) {
        const double detF = d.detF[v];
        double c66[36];
#pragma unroll
        for (int c = 0; c < 36; c++) c66[c] = d.c066mod[c * N + v];
        {
            double Fi[9], g66[36], cm[81], cs[81];
            ld9(d.Finv, N, v, Fi);
            for (int ii = 0; ii < 3; ii++)
                for (int jj = 0; jj < 3; jj++)
                    for (int kk = 0; kk < 3; kk++)
                        for (int ll = 0; ll < 3; ll++) {
                            double dum = 0.0;
                            for (int m = 0; m < 3; m++)
                                for (int n = 0; n < 3; n++) dum += g0[((ii * 3 + m) * 3 + kk) * 3 + n] * Fi[3 * m + jj] * Fi[3 * n + ll];
                            cm[((ii * 3 + jj) * 3 + kk) * 3 + ll] = dum * detF;
                        }
            for (int ii = 0; ii < 3; ii++)
                for (int jj = 0; jj < 3; jj++)
                    for (int kk = 0; kk < 3; kk++)
                        for (int ll = 0; ll < 3; ll++)
                            cs[((ii * 3 + jj) * 3 + kk) * 3 + ll] =
                                0.25 * (cm[((ii * 3 + jj) * 3 + kk) * 3 + ll] + cm[((jj * 3 + ii) * 3 + kk) * 3 + ll] +
                                        cm[((ii * 3 + jj) * 3 + ll) * 3 + kk] + cm[((jj * 3 + ii) * 3 + ll) * 3 + kk]);
            t4_to_b66(cs, g66);
            for (int i = 0; i < 6; i++)
                for (int j = 0; j < 6; j++) {
                    double s = 0.0;
                    for (int k = 0; k < 6; k++) s += c66[6 * i + k] * g66[6 * k + j];
                    d.cG[(6 * i + j) * N + v] = s;
                }
        }
    }
}
void launch_prologue(const Dev& d, const double* c0, const double* goperr0, int do_schmid, int modal, cudaStream_t st) {
    k_prologue<<<d.grid, kBlock, 0, st>>>(d, c0, goperr0, do_schmid, modal);
    if (modal) k_prologue_modal<<<d.grid, kBlock, 0, st>>>(d, goperr0);
}

// ---------------------------------------------------------------- k_gas_compl
__global__ void __launch_bounds__(kBlock) k_gas_compl(Dev d, double tdot, double complgas, int modal) {
    const long long N = d.N;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < N; v += (long long)gridDim.x * blockDim.x) {
        if (!d.gas[v]) {
            for (int c = 0; c < 36; c++) d.cgas[c * N + v] = 0.0;
            continue;
        }
        double a[36];
        for (int i = 0; i < 6; i++)
            for (int j = 0; j < 6; j++) {
                a[6 * i + j] = ((i == j) ? 1.0 : 0.0) + d.c066mod[(6 * i + j) * N + v] / tdot * complgas;
                if (modal) a[6 * i + j] = a[6 * i + j] - d.cG[(6 * i + j) * N + v];
            }
        if (inv_unrolled<6>(a) != 0) set_err(d.err, 1);
        for (int c = 0; c < 36; c++) d.cgas[c * N + v] = a[c];
    }
}
void launch_gas_compl(const Dev& d, double tdot, double complgas, int modal, cudaStream_t st) {
    k_gas_compl<<<d.grid, kBlock, 0, st>>>(d, tdot, complgas, modal);
}

// ---------------------------------------------------------------- k_corr
// velgrad += (dvelgradref + du) F^{-1}; averages; dL statistics; mixing.
// GAS false: a solve without a gas phase (no cgas, no gas voxels), whose gas sums stay zero; the
// kernel then holds eleven fewer running sums and runs without spills (-12 % at 64^3).
template <bool GAS>
__device__ __forceinline__ void body_corr(const Dev& d, const CorrParams& p, const VB& vb) {
    const long long N = d.N;
    __shared__ double du[9];
    if (threadIdx.x < 9) du[threadIdx.x] = __ldcg(&d.red[OFF_DU + threadIdx.x]);
    __syncthreads();
    double s[31];
#pragma unroll
    for (int c = 0; c < 31; c++) s[c] = 0.0;
    for (long long v = vb.x * (long long)blockDim.x + threadIdx.x; v < N; v += (long long)vb.nx * blockDim.x) {
        double t[9], fi[9], u[9], vg[9], vo[9];
        ld9(d.dvr, N, v, t);
        ld9(d.Finv, N, v, fi);
#pragma unroll
        for (int c = 0; c < 9; c++) t[c] = t[c] + du[c];
        mm3(t, fi, u);
        ld9(d.velgrad, N, v, vg);
        ld9(d.velgradold, N, v, vo);
        const double w = d.wgtc[v];
        const bool gas = GAS && d.gas[v];
#pragma unroll
        for (int c = 0; c < 9; c++) {
            vg[c] = vg[c] + u[c];
            s[c] += vg[c] * w;
            if (gas) s[9 + c] += vg[c] * w;
            else s[18 + c] += vg[c] * w;
        }
        if (!p.kinematic) {
            double dl = 0.0;
#pragma unroll
            for (int c = 0; c < 9; c++) dl += (vg[c] - vo[c]) * (vg[c] - vo[c]);
            dl = sqrt(dl);
            double rel = dl / p.Lscale;
            if (gas) { s[29] += (rel * rel) * w; s[30] += w; }
            else { s[27] += (rel * rel) * w; s[28] += w; }
        }
#pragma unroll
        for (int c = 0; c < 9; c++) vg[c] = p.do_mix ? p.mix * vg[c] + (1.0 - p.mix) * vo[c] : p.mix * vg[c];
        st9(d.velgrad, N, v, vg);
        st9(d.velgradold, N, v, vg);
    }
    reduce_store<31, 0>(s, nullptr, d.partials, d.red + OFF_CORR, d.counters + CNT_CORR, vb);
}
__global__ void __launch_bounds__(kBlock, 2) k_corr(Dev d, CorrParams p) {
    if (d.cgas) body_corr<true>(d, p, hw_vb());
    else body_corr<false>(d, p, hw_vb());
}
// fewer blocks than the other voxel kernels: each thread handles several voxels, which spreads the
// 31-field block reduction over more loads
void launch_corr(const Dev& d, const CorrParams& p, cudaStream_t st) {
    const int grid = d.grid < 148 * 2 ? d.grid : 148 * 2;
    k_corr<<<grid, kBlock, 0, st>>>(d, p);
}

// ---------------------------------------------------------------- local constitutive solve
// plastic_strain_rate (various_functions.f90:1367-1419) + elastic_strain_rate (1422-1436)
template <int NS>
__device__ __forceinline__ void constitutive(const PhaseDev& ph, const double* __restrict__ sch, long long N, long long v,
                                             const double (&tt)[NS][2], const double (&sg)[6], double (&edotp)[6],
                                             double (&dd)[15], double (&gamdot)[NS]) {
#pragma unroll
    for (int i = 0; i < 6; i++) edotp[i] = 0.0;
#pragma unroll
    for (int i = 0; i < 15; i++) dd[i] = 0.0;
#pragma unroll
    for (int is = 0; is < NS; is++) {
        if (is < ph.nsyst) {
            double sc[5];
#pragma unroll
            for (int c = 0; c < 5; c++) sc[c] = sch[(is * 5 + c) * N + v];
            double rss = sc[0] * sg[0] + sc[1] * sg[1] + sc[2] * sg[2] + sc[3] * sg[3] + sc[4] * sg[4];
            const double tau = (rss - 0.0 < 0.0) ? tt[is][1] : tt[is][0];  // kin(is) == 0
            rss = (rss - 0.0) / tau;
            const double dum = ph.gamd0[is] * powabs(rss, ph.nrs[is] - 1.0, ph.int_exp);
            const double rss1 = ph.nrs[is] * dum / tau;
            const double rss2 = rss * dum;
            gamdot[is] = rss2;
            int q = 0;
#pragma unroll
            for (int jj = 0; jj < 5; jj++) {
                edotp[jj] = edotp[jj] + sc[jj] * rss2;
#pragma unroll
                for (int ii = 0; ii <= jj; ii++) dd[q++] += sc[ii] * sc[jj] * rss1;
            }
        } else {
            gamdot[is] = 0.0;
        }
    }
}
// x[i] for a run-time i in 0..5 without a local-memory array
__device__ __forceinline__ double sel6(const double (&x)[6], int i) {
    double y = x[0];
#pragma unroll
    for (int c = 1; c < 6; c++) y = (i == c) ? x[c] : y;
    return y;
}
__device__ __forceinline__ double dd_at(const double (&dd)[15], int i, int j) {
    if (i > 4 || j > 4) return 0.0;
    int a = i < j ? i : j, b = i < j ? j : i;
    return dd[b * (b + 1) / 2 + a];
}

// harden (various_functions.f90:1439-1491)
template <int NS>
__device__ __forceinline__ void harden(const PhaseDev& ph, const double* __restrict__ crss, long long N, long long v,
                                       const double (&gamdot)[NS], double gamma0, double tdot, double (&tau)[NS][2], double& gamma1) {
    double deltgam = 0.0;
#pragma unroll
    for (int is = 0; is < NS; is++)
        if (is < ph.nsyst) deltgam = deltgam + fabs(gamdot[is]) * tdot;
    gamma1 = gamma0 + deltgam;
#pragma unroll
    for (int is = 0; is < NS; is++) { tau[is][0] = 0.0; tau[is][1] = 0.0; }
    int is = 0;
    for (int mode = 0; mode < ph.nmodes; mode++) {
        const double tau1 = ph.tau1[mode], thet0 = ph.thet0[mode], thet1 = ph.thet1[mode];
        const double fact = fabs(thet0 / tau1);
        const double exp0 = exp(-fact * gamma0), exp1 = exp(-fact * gamma1);
        const double voce = deltgam * thet1 + tau1 * (exp0 - exp1) + thet1 * (gamma0 * exp0 - gamma1 * exp1);
        for (int ism = 0; ism < ph.nsm[mode]; ism++, is++) {
            double dtau = 0.;
#pragma unroll
            for (int js = 0; js < NS; js++)
                if (js < ph.nsyst) dtau = dtau + ph.hard[is * kMaxSysDev + js] * fabs(gamdot[js]);
#pragma unroll
            for (int q = 0; q < NS; q++)
                if (q == is) {
                    tau[q][0] = crss[(2 * q) * N + v] + dtau * voce * tdot / deltgam;
                    tau[q][1] = crss[(2 * q + 1) * N + v] + dtau * voce * tdot / deltgam;
                }
        }
    }
}

// ---------------------------------------------------------------- k_newton
template <int NS>
__device__ __forceinline__ void body_newton1(const Dev& d, const NewtonParams& p, const VB& vb) {
    const long long N = d.N;
    double s[14];
#pragma unroll
    for (int c = 0; c < 14; c++) s[c] = 0.0;
    for (long long v = vb.x * (long long)blockDim.x + threadIdx.x; v < N; v += (long long)vb.nx * blockDim.x) {
        double lam[6], sg[6], sgt[6], D[6];
        {
            double vg[9], vs[9], a[6];
            ld9(d.velgrad, N, v, vg);
            sym33(vg, vs);
            t2_to_b6(vs, D);
            ld6(d.sg, N, v, a);
            s6_to_b6(a, lam);
            ld6(d.sgt, N, v, a);
            s6_to_b6(a, sgt);
        }
#pragma unroll
        for (int i = 0; i < 6; i++) sg[i] = lam[i];
        const double w = d.wgtc[v];
        if (d.gas[v]) {
            double t[6], res[6], out[6], s6v[6];
#pragma unroll
            for (int i = 0; i < 6; i++) t[i] = D[i] + sgt[i] / p.tdot * p.complgas;
#pragma unroll
            for (int i = 0; i < 6; i++) {
                double a = 0.0;
#pragma unroll
                for (int j = 0; j < 6; j++) a += d.c066mod[(6 * i + j) * N + v] * t[j];
                res[i] = lam[i] + a;
            }
            if (p.modal) {
#pragma unroll
                for (int i = 0; i < 6; i++) {
                    double a = 0.0;
#pragma unroll
                    for (int j = 0; j < 6; j++) a += d.cG[(6 * i + j) * N + v] * lam[j];
                    res[i] -= a;
                }
            }
#pragma unroll
            for (int i = 0; i < 6; i++) {
                double a = 0.0;
#pragma unroll
                for (int j = 0; j < 6; j++) a += d.cgas[(6 * i + j) * N + v] * res[j];
                out[i] = a;
            }
            b6_to_s6(out, s6v);
            st6(d.sg, N, v, s6v);
            double z[6] = {0, 0, 0, 0, 0, 0};
            st6(d.edotp, N, v, z);
            for (int q = 0; q < d.nsys; q++) d.gamdot[q * N + v] = 0.0;
#pragma unroll
            for (int c = 0; c < 6; c++) s[8 + c] += s6v[c] * w;
            continue;
        }
        const PhaseDev& ph = d.ph[d.phase[v]];
        double tt[NS][2];
        double taunrm = 0.0;
#pragma unroll
        for (int q = 0; q < NS; q++) {
            tt[q][0] = (q < d.nsys) ? d.trialtau[(2 * q) * N + v] : 0.0;
            tt[q][1] = (q < d.nsys) ? d.trialtau[(2 * q + 1) * N + v] : 0.0;
            taunrm += tt[q][0] * tt[q][0] + tt[q][1] * tt[q][1];
        }
        taunrm = sqrt(taunrm);
        double edotth[6] = {0, 0, 0, 0, 0, 0};
        if (p.thermo) {
            double e9[9];
            ld9(d.eth, N, v, e9);
            t2_to_b6(e9, edotth);
        }
        double sgnorm = 0.0;
#pragma unroll
        for (int i = 0; i < 6; i++) sgnorm += sg[i] * sg[i];
        sgnorm = sqrt(sgnorm);
        const double tolt = fmax(p.error, p.erroral);
        double errtau = 2.0 * tolt;
        double edotp[6], dd[15], gamdot[NS], edot[6], res[6], sgold[6] = {0, 0, 0, 0, 0, 0};
        double dsgnorm = 0.0, ddgnorm = 0.0;
        const double gamma0 = d.gacumgr[v];
        for (int itertau = 0; itertau < 10 && errtau > tolt;) {
            itertau++;
            int iterNR = 0;
            double erral = 2.0 * p.erroral, resoldn = 1.0;
            while (iterNR < 100 && erral > p.erroral) {
                iterNR++;
                int icut = 0;
                double resn = 2.0 * resoldn;
                while (resn > resoldn && icut < 10) {
                    constitutive<NS>(ph, d.sch, N, v, tt, sg, edotp, dd, gamdot);
                    double ds[6];
#pragma unroll
                    for (int i = 0; i < 6; i++) ds[i] = (sg[i] - sgt[i]) / p.tdot;
#pragma unroll
                    for (int i = 0; i < 6; i++) {
                        double a = 0.0;
#pragma unroll
                        for (int j = 0; j < 6; j++) a += d.sg66[(6 * i + j) * N + v] * ds[j];
                        edot[i] = edotp[i] + a;
                        if (p.thermo) edot[i] = edot[i] + edotth[i];
                    }
#pragma unroll
                    for (int i = 0; i < 6; i++) {
                        double a = 0.0;
#pragma unroll
                        for (int j = 0; j < 6; j++) a += d.c066mod[(6 * i + j) * N + v] * (edot[j] - D[j]);
                        res[i] = sg[i] - lam[i] + a;
                    }
                    if (p.modal) {
                        double r2[6];
#pragma unroll
                        for (int i = 0; i < 6; i++) {
                            double a = 0.0;
#pragma unroll
                            for (int j = 0; j < 6; j++) a += d.cG[(6 * i + j) * N + v] * (sg[j] - lam[j]);
                            r2[i] = a;
                        }
#pragma unroll
                        for (int i = 0; i < 6; i++) res[i] = res[i] - r2[i];
                    }
                    resn = 0.0;
#pragma unroll
                    for (int i = 0; i < 6; i++) resn += res[i] * res[i];
                    resn = sqrt(resn);
                    if (iterNR == 1) resoldn = resn;
                    if (resn > resoldn) {
#pragma unroll
                        for (int i = 0; i < 6; i++) sg[i] = sgold[i] + (sg[i] - sgold[i]) * 0.5;
                    }
                    icut++;
                }
                resoldn = resn;
#pragma unroll
                for (int i = 0; i < 6; i++) sgold[i] = sg[i];
                double J[36];
#pragma unroll
                for (int i = 0; i < 6; i++) {
                    double crow[6];
#pragma unroll
                    for (int k = 0; k < 6; k++) crow[k] = d.c066mod[(6 * i + k) * N + v];
#pragma unroll
                    for (int j = 0; j < 6; j++) {
                        double a = 0.0;
#pragma unroll
                        for (int k = 0; k < 6; k++) a += crow[k] * (dd_at(dd, k, j) + d.sg66[(6 * k + j) * N + v] / p.tdot);
                        J[6 * i + j] = ((i == j) ? 1.0 : 0.0) + a;
                        if (p.modal) J[6 * i + j] -= d.cG[(6 * i + j) * N + v];
                    }
                }
                if (solve6(J, res) != 0) set_err(d.err, 1);
                double a = 0.0, b = 0.0, c = 0.0;
#pragma unroll
                for (int i = 0; i < 6; i++) {
                    sg[i] = sg[i] - res[i];
                    a += (sg[i] - sgold[i]) * (sg[i] - sgold[i]);
                    b += (sg[i] - lam[i]) * (sg[i] - lam[i]);
                    c += (edot[i] - D[i]) * (edot[i] - D[i]);
                }
                dsgnorm = b;
                ddgnorm = c;
                erral = sqrt(a) / sgnorm;
            }
            if (p.iuphard) {
                double tn[NS][2], g1;
                harden<NS>(ph, d.crss, N, v, gamdot, gamma0, p.tdot, tn, g1);
                double e2 = 0.0;
#pragma unroll
                for (int q = 0; q < NS; q++) {
                    e2 += (tt[q][0] - tn[q][0]) * (tt[q][0] - tn[q][0]) + (tt[q][1] - tn[q][1]) * (tt[q][1] - tn[q][1]);
                    tt[q][0] = tn[q][0];
                    tt[q][1] = tn[q][1];
                }
                errtau = sqrt(e2) / taunrm;
            } else {
                errtau = 0.0;
            }
        }
        double s6v[6], e6v[6];
        b6_to_s6(sg, s6v);
        b6_to_s6(edotp, e6v);
        st6(d.sg, N, v, s6v);
        st6(d.edotp, N, v, e6v);
#pragma unroll
        for (int q = 0; q < NS; q++)
            if (q < d.nsys) {
                d.gamdot[q * N + v] = gamdot[q];
                d.trialtau[(2 * q) * N + v] = tt[q][0];
                d.trialtau[(2 * q + 1) * N + v] = tt[q][1];
            }
        if (!(dsgnorm == dsgnorm) || !(ddgnorm == ddgnorm)) set_err(d.err, 2);
        s[0] += dsgnorm * w;
        s[1] += ddgnorm * w;
#pragma unroll
        for (int c = 0; c < 6; c++) {
            s[2 + c] += w * s6v[c];
            s[8 + c] += s6v[c] * w;
        }
    }
    reduce_store<14, 0>(s, nullptr, d.partials, d.red + OFF_NEWTON, d.counters + CNT_NEWTON, vb);
}
template <int NS>
__global__ void __launch_bounds__(kNewtonBlock, 2) k_newton(Dev d, NewtonParams p) { body_newton1<NS>(d, p, hw_vb()); }
// ---------------------------------------------------------------- k_newton6: six lanes per voxel
// The local solve of k_newton with the voxel's operators held in registers for
// the whole Newton solve instead of being re-read from memory at every
// evaluation.  A warp holds five voxels, one per group of six lanes (lanes 30
// and 31 hold none).  Lane r of a group owns row r of C~ (c066mod), of the
// compliance S (sg66), of M = C~ S / dt and, with the augmented Lagrangian,
// of C~ Gamma (cG); it owns component r of every 6-vector in the b-basis and
// the slip systems s = r + 6k.  Vectors are exchanged with warp shuffles and
// group sums are formed in one fixed order, so every lane of a group holds the
// bitwise-identical sum.  All loops run warp-uniformly (until no group of the
// warp is still active), with every state update predicated on its group's
// flag, so the shuffles always use the full warp mask.  The 6x6 Newton system
// is solved by Gauss-Jordan elimination with partial pivoting (pivot: largest
// |a| in the column, first row on ties, as dgesv), one row per lane, without
// moving rows between lanes.  Against k_newton the arithmetic differs only in
// rounding: the Jacobian is I + C~ dd + M (- cG), sums run in another order
// and the elimination is Gauss-Jordan.
constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ double gsum6(double x, int base) {
    const double pr = x + __shfl_xor_sync(kFull, x, 1);  // lanes 2j, 2j+1 of a group (groups start at even lanes)
    const double p0 = __shfl_sync(kFull, pr, base), p1 = __shfl_sync(kFull, pr, base + 2),
                 p2 = __shfl_sync(kFull, pr, base + 4);
    return (p0 + p1) + p2;
}
__device__ __forceinline__ unsigned long long umax64(unsigned long long a, unsigned long long b) { return a > b ? a : b; }

// Per-warp shared memory: rows of kXStride doubles, one double per lane (33 so that
// lanes reading other lanes' entries hit distinct banks).
constexpr int kXRows = 16, kXStride = 33;
// N doubles owned by a lane: a column of the warp's shared memory (entries kXStride
// apart) when SM, else registers (every index must then be a compile-time constant).
template <bool SM, int N>
struct LaneCol {
    double* p;
    double r[SM ? 1 : N];
    __device__ __forceinline__ double& operator[](int i) {
        if constexpr (SM) return p[i * kXStride];
        else return r[i];
    }
};

// Dynamic shared memory of k_newton6: with two systems per lane, per warp the lanes' Schmid
// vectors (5 * SPL), rows of C~ and A (12), trial resistances (2 * SPL), slip rates, rate
// factors, rate constants and exponents (4 * SPL) as columns; nothing with four per lane.
__host__ __device__ constexpr bool newton6_cols_in_smem(int spl) { return spl == 2; }
__host__ __device__ constexpr int newton6_col_rows(int spl) { return newton6_cols_in_smem(spl) ? 11 * spl + 12 : 0; }
__host__ __device__ constexpr size_t newton6_smem_bytes(int spl) {
    return 8 * sizeof(double) * (size_t)newton6_col_rows(spl) * kXStride;
}

template <int SPL, bool MODAL>
__device__ __forceinline__ void body_newton6(const Dev& d, const NewtonParams& p, const VB& vb) {
    constexpr bool kSm = newton6_cols_in_smem(SPL);
    extern __shared__ double dyn_smem[];
    double* const col = dyn_smem + (threadIdx.x >> 5) * newton6_col_rows(SPL) * kXStride + (threadIdx.x & 31);
    LaneCol<kSm, 6> Crow{col}, Arow{col + 6 * kXStride};             // rows r of C~ and A
    LaneCol<kSm, 5 * SPL> SCH{col + 12 * kXStride};                  // Schmid vectors of the lane's systems
    LaneCol<kSm, 2 * SPL> TT{col + (12 + 5 * SPL) * kXStride};       // trial resistances
    LaneCol<kSm, SPL> GD{col + (12 + 7 * SPL) * kXStride};           // accepted slip rates
    LaneCol<kSm, SPL> RS{col + (12 + 8 * SPL) * kXStride};           // and rate factors
    LaneCol<kSm, SPL> G0{col + (12 + 9 * SPL) * kXStride};           // reference rates
    LaneCol<kSm, SPL> NR{col + (12 + 10 * SPL) * kXStride};          // rate exponents
    const long long N = d.N;
    const int lane = threadIdx.x & 31;
    const int grp = lane / 6;               // 0..4 hold voxels; group 5 (lanes 30, 31) is idle
    const int r = lane - 6 * grp;           // row / component owned by this lane
    const int base = grp < 5 ? 6 * grp : 24;  // idle lanes shadow group 4's lanes and write nothing
    double acc[14];
#pragma unroll
    for (int c = 0; c < 14; c++) acc[c] = 0.0;
    const long long wid = ((long long)vb.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarp = ((long long)vb.nx * blockDim.x) >> 5;
    const double tolt = fmax(p.error, p.erroral);
    for (long long v0 = wid * 5; v0 < N; v0 += nwarp * 5) {  // warp-uniform
        const bool valid = grp < 5 && v0 + grp < N;
        const long long v = valid ? v0 + grp : v0;  // in-range index for the loads of idle lanes
        const bool gas = valid && d.gas[v];
        const bool act = valid && !gas;
        const double w = d.wgtc[v];
        if (gas && r == 0) {  // dummy gas voxel: closed-form update by one lane
            double lam[6], sgt6[6], D6[6], t[6], res[6], out[6], s6v[6], a[6], vg[9], vs[9];
            ld6(d.sg, N, v, a);
            s6_to_b6(a, lam);
            ld6(d.sgt, N, v, a);
            s6_to_b6(a, sgt6);
            ld9(d.velgrad, N, v, vg);
            sym33(vg, vs);
            t2_to_b6(vs, D6);
#pragma unroll
            for (int i = 0; i < 6; i++) t[i] = D6[i] + sgt6[i] / p.tdot * p.complgas;
#pragma unroll
            for (int i = 0; i < 6; i++) {
                double x = 0.0;
#pragma unroll
                for (int j = 0; j < 6; j++) x += d.c066mod[(6 * i + j) * N + v] * t[j];
                res[i] = lam[i] + x;
            }
            if (MODAL) {
#pragma unroll
                for (int i = 0; i < 6; i++) {
                    double x = 0.0;
#pragma unroll
                    for (int j = 0; j < 6; j++) x += d.cG[(6 * i + j) * N + v] * lam[j];
                    res[i] -= x;
                }
            }
#pragma unroll
            for (int i = 0; i < 6; i++) {
                double x = 0.0;
#pragma unroll
                for (int j = 0; j < 6; j++) x += d.cgas[(6 * i + j) * N + v] * res[j];
                out[i] = x;
            }
            b6_to_s6(out, s6v);
            st6(d.sg, N, v, s6v);
#pragma unroll
            for (int c = 0; c < 6; c++) d.edotp[c * N + v] = 0.0;
            for (int q = 0; q < d.nsys; q++) d.gamdot[q * N + v] = 0.0;
#pragma unroll
            for (int c = 0; c < 6; c++) acc[8 + c] += s6v[c] * w;
        }
        // per-voxel vectors: full in every lane while A and q are formed, component r afterwards
        double lam_r, sgt_r, D_r, eth_r, q_r;
        const PhaseDev& ph = d.ph[d.phase[v]];
        const int nsyst = ph.nsyst;
        {
        double lamf[6], sgtf[6], Df[6], ethf[6] = {0, 0, 0, 0, 0, 0};
        {
            double a[9], vs[9];
            ld6(d.sg, N, v, a);
            s6_to_b6(a, lamf);
            ld6(d.sgt, N, v, a);
            s6_to_b6(a, sgtf);
            ld9(d.velgrad, N, v, a);
            sym33(a, vs);
            t2_to_b6(vs, Df);
            if (p.thermo) {
                ld9(d.eth, N, v, a);
                t2_to_b6(a, ethf);
            }
        }
        // The residual of solve_res,
        //   res = sg - lam + C~ (edotp + S (sg - sgt) / dt + eth - D) - cG (sg - lam),
        // is evaluated as res = A sg + C~ edotp - q with, per voxel,
        //   A = I + M - cG,  M = C~ S / dt,  q = lam + M sgt + C~ (D - eth) - cG lam,
        // and the Jacobian is A + C~ dd.  Lane r keeps rows r of C~ and A and q_r.
        {
            double Srow[6], M[6];
#pragma unroll
            for (int j = 0; j < 6; j++) {
                Crow[j] = d.c066mod[(6 * r + j) * N + v];
                Srow[j] = d.sg66[(6 * r + j) * N + v];
                M[j] = 0.0;
            }
#pragma unroll
            for (int k = 0; k < 6; k++)
#pragma unroll
                for (int j = 0; j < 6; j++) M[j] += Crow[k] * (__shfl_sync(kFull, Srow[j], base + k) / p.tdot);
            q_r = sel6(lamf, r);
            double ms = 0.0, cd = 0.0, gl = 0.0;
#pragma unroll
            for (int j = 0; j < 6; j++) {
                const double g = MODAL ? d.cG[(6 * r + j) * N + v] : 0.0;
                Arow[j] = ((r == j) ? 1.0 : 0.0) + M[j] - g;
                ms += M[j] * sgtf[j];
                cd += Crow[j] * (Df[j] - ethf[j]);
                gl += g * lamf[j];
            }
            q_r = q_r + ms + cd - gl;
        }
        lam_r = sel6(lamf, r);
        sgt_r = sel6(sgtf, r);
        D_r = sel6(Df, r);
        eth_r = sel6(ethf, r);
        }
        // slip systems of this lane and their constants
        double taun = 0.0;
#pragma unroll
        for (int k = 0; k < SPL; k++) {
            const int s = r + 6 * k;
            const bool own = s < nsyst, any = s < d.nsys;
#pragma unroll
            for (int c = 0; c < 5; c++) SCH[5 * k + c] = own ? d.sch[(s * 5 + c) * N + v] : 0.0;
            TT[2 * k] = any ? d.trialtau[(2 * s) * N + v] : 0.0;
            TT[2 * k + 1] = any ? d.trialtau[(2 * s + 1) * N + v] : 0.0;
            G0[k] = own ? ph.gamd0[s] : 0.0;
            NR[k] = own ? ph.nrs[s] : 1.0;
            GD[k] = 0.0;
            RS[k] = 0.0;
            taun += TT[2 * k] * TT[2 * k] + TT[2 * k + 1] * TT[2 * k + 1];
        }
        const int int_exp = ph.int_exp;
        taun = sqrt(gsum6(taun, base));
        double sg_r = lam_r;
        const double sgnorm = sqrt(gsum6(sg_r * sg_r, base));
        double sgold_r = 0.0, sev_r = 0.0, edotp_r = 0.0;
        const double gamma0 = d.gacumgr[v];
        int itertau = 0;
        double errtau = 2.0 * tolt;
        bool aT = act;
        while (true) {
            aT = aT && itertau < 10 && errtau > tolt;
            if (!__any_sync(kFull, aT)) break;
            itertau += aT;
            int iterNR = 0;
            double erral = 2.0 * p.erroral, resoldn = 1.0;
            bool aN = aT;
            while (true) {
                aN = aN && iterNR < 100 && erral > p.erroral;
                if (!__any_sync(kFull, aN)) break;
                iterNR += aN;
                int icut = 0;
                double resn = 2.0 * resoldn, res_r = 0.0;
                bool aC = aN;
                while (true) {
                    aC = aC && resn > resoldn && icut < 10;
                    if (!__any_sync(kFull, aC)) break;
                    // plastic_strain_rate at sg (own systems), summed over the group
                    double sgf[6];
#pragma unroll
                    for (int c = 0; c < 6; c++) sgf[c] = __shfl_sync(kFull, sg_r, base + c);
                    double ep[5] = {0, 0, 0, 0, 0}, gdn[SPL], rsn[SPL];
#pragma unroll
                    for (int k = 0; k < SPL; k++) {
                        gdn[k] = 0.0;
                        rsn[k] = 0.0;
                        if (r + 6 * k < nsyst) {
                            double rss = SCH[5 * k + 0] * sgf[0] + SCH[5 * k + 1] * sgf[1] + SCH[5 * k + 2] * sgf[2] + SCH[5 * k + 3] * sgf[3] +
                                         SCH[5 * k + 4] * sgf[4];
                            const double tau = (rss - 0.0 < 0.0) ? TT[2 * k + 1] : TT[2 * k];
                            rss = (rss - 0.0) / tau;
                            const double dum = G0[k] * powabs(rss, NR[k] - 1.0, int_exp);
                            rsn[k] = NR[k] * dum / tau;
                            gdn[k] = rss * dum;
#pragma unroll
                            for (int c = 0; c < 5; c++) ep[c] += SCH[5 * k + c] * gdn[k];
                        }
                    }
                    double rn = -q_r, epr = 0.0;
#pragma unroll
                    for (int c = 0; c < 5; c++) {
                        const double t = gsum6(ep[c], base);
                        epr = (r == c) ? t : epr;
                        rn += Crow[c] * t;
                    }
#pragma unroll
                    for (int j = 0; j < 6; j++) rn += Arow[j] * sgf[j];
                    const double rnn = sqrt(gsum6(rn * rn, base));
                    if (aC) {
#pragma unroll
                        for (int k = 0; k < SPL; k++) {
                            GD[k] = gdn[k];
                            RS[k] = rsn[k];
                        }
                        edotp_r = epr;
                        sev_r = sg_r;
                        res_r = rn;
                        resn = rnn;
                        if (iterNR == 1) resoldn = resn;
                        if (resn > resoldn) sg_r = sgold_r + (sg_r - sgold_r) * 0.5;
                        icut++;
                    }
                }
                if (aN) {
                    resoldn = resn;
                    sgold_r = sg_r;
                }
                // d(edotp)/d(sigma): the 5x5 symmetric sum over the group's systems
                double dd[15];
#pragma unroll
                for (int q = 0; q < 15; q++) dd[q] = 0.0;
#pragma unroll
                for (int k = 0; k < SPL; k++) {
                    if (r + 6 * k < nsyst) {
                        int q = 0;
#pragma unroll
                        for (int jj = 0; jj < 5; jj++)
#pragma unroll
                            for (int ii = 0; ii <= jj; ii++) dd[q++] += SCH[5 * k + ii] * SCH[5 * k + jj] * RS[k];
                    }
                }
#pragma unroll
                for (int q = 0; q < 15; q++) dd[q] = gsum6(dd[q], base);
                // row r of the Jacobian A + C~ dd
                double Jr[6];
#pragma unroll
                for (int j = 0; j < 6; j++) {
                    double x = 0.0;
#pragma unroll
                    for (int k = 0; k < 5; k++) x += Crow[k] * dd_at(dd, k, j);
                    Jr[j] = Arow[j] + x;
                }
                // Gauss-Jordan elimination; the low three bits of the pivot key carry 7 - row
                double b = res_r, dpiv = 1.0;
                bool sing = false;
                unsigned usedm = 0u;  // rows already pivoted (group-uniform)
                int pvs[6];
#pragma unroll
                for (int k = 0; k < 6; k++) {
                    int pv;
                    if (k < 5) {
                        unsigned long long key =
                            ((usedm >> r) & 1u)
                                ? 0ull
                                : (((unsigned long long)__double_as_longlong(fabs(Jr[k])) & ~7ull) | (unsigned long long)(7 - r));
                        key = umax64(key, __shfl_xor_sync(kFull, key, 1));
                        key = umax64(umax64(__shfl_sync(kFull, key, base), __shfl_sync(kFull, key, base + 2)),
                                     __shfl_sync(kFull, key, base + 4));
                        pv = 7 - (int)(key & 7ull);
                    } else {
                        pv = __ffs(~usedm & 63u) - 1;  // the one row left
                    }
                    pvs[k] = pv;
                    usedm |= 1u << pv;
                    const bool me = (r == pv);
                    double pk[6];
#pragma unroll
                    for (int j = k; j < 6; j++) pk[j] = __shfl_sync(kFull, Jr[j], base + pv);
                    const double bk = __shfl_sync(kFull, b, base + pv);
                    sing = sing || (pk[k] == 0.0);
                    const double rinv = 1.0 / pk[k];
                    if (me) {
                        dpiv = pk[k];
                    } else {
                        const double l = Jr[k] * rinv;
#pragma unroll
                        for (int j = k + 1; j < 6; j++) Jr[j] -= l * pk[j];
                        b -= l * bk;
                    }
                }
                // this lane's row now gives the unknown of the column it pivoted; fetch component r
                const double xown = b / dpiv;
                int src = pvs[0];
#pragma unroll
                for (int k = 1; k < 6; k++) src = (r == k) ? pvs[k] : src;
                const double xr = __shfl_sync(kFull, xown, base + src);
                const double sg_new = sg_r - xr;
                const double dsgnr = gsum6((sg_new - sgold_r) * (sg_new - sgold_r), base);
                if (aN) {
                    if (sing && r == 0) set_err(d.err, 1);
                    sg_r = sg_new;
                    erral = sqrt(dsgnr) / sgnorm;
                }
            }
            if (p.iuphard) {  // harden (various_functions.f90:1439-1491)
                double dg = 0.0;
#pragma unroll
                for (int k = 0; k < SPL; k++)
                    if (r + 6 * k < nsyst) dg += fabs(GD[k]) * p.tdot;
                const double deltgam = gsum6(dg, base);
                const double gamma1 = gamma0 + deltgam;
                double gall[6 * SPL];
#pragma unroll
                for (int k = 0; k < SPL; k++)
#pragma unroll
                    for (int q = 0; q < 6; q++) gall[6 * k + q] = fabs(__shfl_sync(kFull, GD[k], base + q));
                double e2 = 0.0, tn[SPL][2];
#pragma unroll
                for (int k = 0; k < SPL; k++) {
                    const int s = r + 6 * k;
                    tn[k][0] = 0.0;  // systems beyond the phase's own get zero resistance, as harden leaves them
                    tn[k][1] = 0.0;
                    if (s < nsyst) {
                        int mode = 0, last = ph.nsm[0];
                        while (mode + 1 < ph.nmodes && s >= last) {
                            mode++;
                            last += ph.nsm[mode];
                        }
                        const double tau1 = ph.tau1[mode], thet0 = ph.thet0[mode], thet1 = ph.thet1[mode];
                        const double fact = fabs(thet0 / tau1);
                        const double exp0 = exp(-fact * gamma0), exp1 = exp(-fact * gamma1);
                        const double voce =
                            deltgam * thet1 + tau1 * (exp0 - exp1) + thet1 * (gamma0 * exp0 - gamma1 * exp1);
                        double dtau = 0.0;
#pragma unroll
                        for (int js = 0; js < 6 * SPL; js++)
                            if (js < nsyst) dtau = dtau + ph.hard[s * kMaxSysDev + js] * gall[js];
                        tn[k][0] = d.crss[(2 * s) * N + v] + dtau * voce * p.tdot / deltgam;
                        tn[k][1] = d.crss[(2 * s + 1) * N + v] + dtau * voce * p.tdot / deltgam;
                    }
                    e2 += (TT[2 * k] - tn[k][0]) * (TT[2 * k] - tn[k][0]) + (TT[2 * k + 1] - tn[k][1]) * (TT[2 * k + 1] - tn[k][1]);
                }
                const double et = sqrt(gsum6(e2, base)) / taun;
                if (aT) {
#pragma unroll
                    for (int k = 0; k < SPL; k++) {
                        TT[2 * k] = tn[k][0];
                        TT[2 * k + 1] = tn[k][1];
                    }
                    errtau = et;
                }
            } else if (aT) {
                errtau = 0.0;
            }
        }
        // |sg - lam|^2 at the final stress; |edot - D|^2 at the last evaluation, with
        // edot = edotp + S (sg - sgt) / dt + eth as elastic_strain_rate forms it
        double sgf[6], epf[6], ee = 0.0;
        {
            const double ds_r = (sev_r - sgt_r) / p.tdot;
#pragma unroll
            for (int j = 0; j < 6; j++) ee += d.sg66[(6 * r + j) * N + v] * __shfl_sync(kFull, ds_r, base + j);
        }
        double edot_r = edotp_r + ee;
        if (p.thermo) edot_r = edot_r + eth_r;
        const double dl = sg_r - lam_r, de = edot_r - D_r;
        const double dsgnorm = gsum6(dl * dl, base), ddgnorm = gsum6(de * de, base);
        // outputs: sigma and edotp in the symmetric 3x3 form, slip rates and resistances
#pragma unroll
        for (int c = 0; c < 6; c++) {
            sgf[c] = __shfl_sync(kFull, sg_r, base + c);
            epf[c] = __shfl_sync(kFull, edotp_r, base + c);
        }
        epf[5] = 0.0;
        if (act) {
            double s6v[6], e6v[6];
            b6_to_s6(sgf, s6v);
            b6_to_s6(epf, e6v);
            d.sg[r * N + v] = sel6(s6v, r);
            d.edotp[r * N + v] = sel6(e6v, r);
#pragma unroll
            for (int k = 0; k < SPL; k++) {
                const int s = r + 6 * k;
                if (s < d.nsys) {
                    d.gamdot[s * N + v] = (s < nsyst) ? GD[k] : 0.0;
                    d.trialtau[(2 * s) * N + v] = TT[2 * k];
                    d.trialtau[(2 * s + 1) * N + v] = TT[2 * k + 1];
                }
            }
            if (r == 0) {
                if (!(dsgnorm == dsgnorm) || !(ddgnorm == ddgnorm)) set_err(d.err, 2);
                acc[0] += dsgnorm * w;
                acc[1] += ddgnorm * w;
#pragma unroll
                for (int c = 0; c < 6; c++) {
                    acc[2 + c] += w * s6v[c];
                    acc[8 + c] += s6v[c] * w;
                }
            }
        }
    }
    reduce_store<14, 0>(acc, nullptr, d.partials, d.red + OFF_NEWTON, d.counters + CNT_NEWTON, vb);
}

// ---------------------------------------------------------------- shared-memory exchange of k_newton6p
// Group sums and broadcasts go through a per-warp area of shared memory (one
// 64-bit store or load per double, where a shuffle moves 32 bits).  Rows hold
// one double per lane at a stride of 33 doubles, so that lanes reading another
// lane's entries hit distinct banks.  Every write phase starts with
// __syncwarp(), so a row is never overwritten before all lanes have read it.
struct Xw {
    double* P;      // [kXRows][kXStride]; row kXRows - 1 serves the scalar sums and gathers
    int lane, base;
};
// group sum in lane order, identical in every lane of the group
__device__ __forceinline__ double xsum(const Xw& X, double x) {
    double* row = X.P + (kXRows - 1) * kXStride;
    __syncwarp();
    row[X.lane] = x;
    __syncwarp();
    const double* q = row + X.base;
    return ((((q[0] + q[1]) + q[2]) + q[3]) + q[4]) + q[5];
}
// the group's six values of x, in every lane of the group
__device__ __forceinline__ void xgather(const Xw& X, double x, double (&out)[6]) {
    double* row = X.P + (kXRows - 1) * kXStride;
    __syncwarp();
    row[X.lane] = x;
    __syncwarp();
#pragma unroll
    for (int c = 0; c < 6; c++) out[c] = row[X.base + c];
}

template <int SPL, bool MODAL>
__global__ void __launch_bounds__(256, 2) k_newton6(Dev d, NewtonParams p) { body_newton6<SPL, MODAL>(d, p, hw_vb()); }

// What the local solve reads of a phase, staged in shared memory once per block
// (MS systems at most: 12 or 24).
template <int MS>
struct PhaseN {
    int nsyst, nmodes, int_exp, nsm[3];
    double nrs[MS], gamd0[MS];
    double tau1[3], thet0[3], thet1[3];
    double hard[MS * MS];
};
constexpr int kMaxPhaseSmem = 4;


// Dynamic shared memory of k_newton6p: the staged phases, then per warp the
// exchange rows, the lanes' columns (rows of kXStride doubles) and the five
// groups' sums (70).  The columns hold the Schmid vectors (5 * SPL) and, with
// two systems per lane (12-system phases), also the lane's rows of C~ and H0
// (12), its trial resistances (2 * SPL), accepted slip rates and rate factors
// (2 * SPL) and three stress/strain-rate components: kept out of registers,
// they leave the Newton loop nearly free of spills, and two blocks of 256
// threads still fit one SM.  With four systems per lane those stay in registers
// (the larger columns would leave room for one block per SM).
__host__ __device__ constexpr bool newton6p_cols_in_smem(int spl) { return spl == 2; }
__host__ __device__ constexpr int newton6p_col_rows(int spl) {
    return 5 * spl + (newton6p_cols_in_smem(spl) ? 12 + 4 * spl + 3 : 0);
}
__host__ __device__ constexpr int newton6p_warp_doubles(int spl) {
    return kXRows * kXStride + newton6p_col_rows(spl) * kXStride + 70;
}
__host__ __device__ constexpr size_t newton6p_smem_bytes(int spl, int nph) {
    return (size_t)nph * (spl == 2 ? sizeof(PhaseN<12>) : sizeof(PhaseN<24>)) +
           8 * sizeof(double) * (size_t)newton6p_warp_doubles(spl);
}

// ---------------------------------------------------------------- k_newton6p: symmetric positive definite form
// The local solve without the augmented-Lagrangian term (the modal path uses
// k_newton6), with the Newton system put in symmetric form.  With
// dedot = dd + S / dt the Jacobian of solve_res is
//   J = I + C~ (S / dt + dd) = C~ H,   H = C~^-1 + S / dt + dd,
// where C~ (c066mod) and S (sg66) are symmetric positive definite and dd is
// positive semi-definite, so H is symmetric positive definite.  The Newton
// step J^-1 res equals H^-1 rho with rho = C~^-1 res, and rho is formed
// directly:
//   rho = H0 sg + edotp - q',  H0 = C~^-1 + S / dt,  q' = C~^-1 lam + (S / dt) sgt + D - eth,
// while res = C~ rho gives the residual norm that drives the step halving.
// Elimination on H needs no pivoting: lanes eliminate in the fixed order
// 0..5 (Gauss-Jordan), and lane r ends with the unknown of column r; lane r
// reads only row r of dd.  Against dgesv on J the Newton step differs in
// rounding only.  Five voxels per warp, six lanes per voxel as in k_newton6;
// the Schmid vectors, the per-group sums and (two systems per lane) the lane's
// operator rows and per-system state live in shared memory, which keeps the
// kernel within 128 registers with few spills (16 warps per SM).
template <int SPL>
__device__ __forceinline__ void body_newton6p(const Dev& d, const NewtonParams& p, const VB& vb) {
    constexpr int MS = 6 * SPL;
    constexpr bool kSm = newton6p_cols_in_smem(SPL);
    extern __shared__ double dyn_smem[];
    PhaseN<MS>* const sph = reinterpret_cast<PhaseN<MS>*>(dyn_smem);
    const int nph = d.nph < kMaxPhaseSmem ? d.nph : kMaxPhaseSmem;
    for (int q = threadIdx.x; q < nph; q += blockDim.x) {
        const PhaseDev& g = d.ph[q];
        sph[q].nsyst = g.nsyst;
        sph[q].nmodes = g.nmodes;
        sph[q].int_exp = g.int_exp;
        for (int m = 0; m < 3; m++) {
            sph[q].nsm[m] = g.nsm[m];
            sph[q].tau1[m] = g.tau1[m];
            sph[q].thet0[m] = g.thet0[m];
            sph[q].thet1[m] = g.thet1[m];
        }
    }
    for (int e = threadIdx.x; e < nph * MS; e += blockDim.x) {
        sph[e / MS].nrs[e % MS] = d.ph[e / MS].nrs[e % MS];
        sph[e / MS].gamd0[e % MS] = d.ph[e / MS].gamd0[e % MS];
    }
    for (int e = threadIdx.x; e < nph * MS * MS; e += blockDim.x) {
        const int q = e / (MS * MS), i = (e % (MS * MS)) / MS, j = e % MS;
        sph[q].hard[i * MS + j] = d.ph[q].hard[i * kMaxSysDev + j];
    }
    __syncthreads();
    double* const wsm = reinterpret_cast<double*>(sph + nph) + (threadIdx.x >> 5) * newton6p_warp_doubles(SPL);
    const long long N = d.N;
    const int lane = threadIdx.x & 31;
    const int grp = lane / 6;                 // 0..4 hold voxels; group 5 (lanes 30, 31) is idle
    const int r = lane - 6 * grp;             // row / component owned by this lane
    const int base = grp < 5 ? 6 * grp : 24;  // idle lanes shadow group 4's lanes and write nothing
    const Xw X{wsm, lane, base};
    // this lane's column: Schmid vectors, then (kSm) the values below
    double* const schm = wsm + kXRows * kXStride + lane;
    double* const col = schm + 5 * SPL * kXStride;
    LaneCol<kSm, 6> Crow{col}, Hrow{col + 6 * kXStride};    // rows r of C~ and H0
    LaneCol<kSm, 2 * SPL> TT{col + 12 * kXStride};          // trial resistances of the lane's systems
    LaneCol<kSm, SPL> GD{col + (12 + 2 * SPL) * kXStride};  // accepted slip rates
    LaneCol<kSm, SPL> RS{col + (12 + 3 * SPL) * kXStride};  // and their d(rate)/d(tau) factors
    LaneCol<kSm, 1> LAM{col + (12 + 4 * SPL) * kXStride};   // component r of the input stress,
    LaneCol<kSm, 1> SEV{col + (13 + 4 * SPL) * kXStride};   // of the stress at the last accepted evaluation
    LaneCol<kSm, 1> EPM{col + (14 + 4 * SPL) * kXStride};   // and of the plastic strain rate there
    double* const accw = wsm + kXRows * kXStride + newton6p_col_rows(SPL) * kXStride;
    for (int c = lane; c < 70; c += 32) accw[c] = 0.0;
    __syncwarp();
    double* const accg = accw + (grp < 5 ? grp : 0) * 14;
    const double tolt = fmax(p.error, p.erroral);
    const long long wid = ((long long)vb.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarp = ((long long)vb.nx * blockDim.x) >> 5;
    const bool stats = d.nstats != nullptr;
    unsigned long long c_pass = 0, c_eval = 0, c_nr = 0, c_tau = 0, c_vox = 0, c_npass = 0;  // warp-uniform counts
    const unsigned lead = 0x01041041u;  // lanes 0, 6, 12, 18, 24: one per voxel group
    for (long long v0 = wid * 5; v0 < N; v0 += nwarp * 5) {  // warp-uniform
        const bool valid = grp < 5 && v0 + grp < N;
        const long long v = valid ? v0 + grp : v0;  // in-range index for the loads of idle lanes
        const bool gasv = d.gas[v];
        const int phi = d.phase[v];
        // rows r of C~ and H0, q'_r and this lane's systems; no load waits on the gas flag or phase
        double qp_r, sgt_r, D_r, eth_r = 0.0;  // component r of sgt, of D and of eth: kept for the closing norms
        {
            double lamf[6], sgtf[6], a[9], b6[6], vs[9];
            ld6(d.sg, N, v, a);
            s6_to_b6(a, lamf);
            ld6(d.sgt, N, v, a);
            s6_to_b6(a, sgtf);
            sgt_r = sel6(sgtf, r);
            ld9(d.velgrad, N, v, a);
            sym33(a, vs);
            t2_to_b6(vs, b6);
            D_r = sel6(b6, r);
            double De = D_r;
            if (p.thermo) {
                ld9(d.eth, N, v, a);
                t2_to_b6(a, b6);
                eth_r = sel6(b6, r);
                De = De - eth_r;
            }
            double cl = 0.0, ss = 0.0;
#pragma unroll
            for (int j = 0; j < 6; j++) {
                Crow[j] = d.c066mod[(6 * r + j) * N + v];
                const double ci = d.c066inv[(6 * r + j) * N + v];
                const double sd = d.sg66[(6 * r + j) * N + v] / p.tdot;
                Hrow[j] = ci + sd;
                cl += ci * lamf[j];
                ss += sd * sgtf[j];
            }
            qp_r = cl + ss + De;
            LAM[0] = sel6(lamf, r);
#pragma unroll
            for (int k = 0; k < SPL; k++) {
                const int s = r + 6 * k;
                const bool any = s < d.nsys;
#pragma unroll
                for (int c = 0; c < 5; c++) schm[(5 * k + c) * kXStride] = any ? d.sch[(s * 5 + c) * N + v] : 0.0;
                TT[2 * k] = any ? d.trialtau[(2 * s) * N + v] : 0.0;
                TT[2 * k + 1] = any ? d.trialtau[(2 * s + 1) * N + v] : 0.0;
            }
        }
        const PhaseN<MS>& ph = sph[phi];
        const int nsyst = ph.nsyst;
        const bool gas = valid && gasv;
        const bool act = valid && !gas;

        double taun = 0.0;
#pragma unroll
        for (int k = 0; k < SPL; k++) {
            const int s = r + 6 * k;
            const bool own = s < nsyst;
            if (!own)
#pragma unroll
                for (int c = 0; c < 5; c++) schm[(5 * k + c) * kXStride] = 0.0;
            GD[k] = 0.0;
            RS[k] = 0.0;
            const double t0 = TT[2 * k], t1 = TT[2 * k + 1];
            taun += t0 * t0 + t1 * t1;
        }
        const int int_exp = ph.int_exp;
        taun = sqrt(xsum(X, taun));
        double sg_r = LAM[0];
        const double sgnorm = sqrt(xsum(X, sg_r * sg_r));
        double sgold_r = 0.0;
        SEV[0] = 0.0;
        EPM[0] = 0.0;
        int itertau = 0;
        double errtau = 2.0 * tolt;
        bool aT = act;
        if (stats) c_vox += __popc(__ballot_sync(kFull, act) & lead);
        while (true) {
            aT = aT && itertau < 10 && errtau > tolt;
            if (!__any_sync(kFull, aT)) break;
            if (stats) c_tau += __popc(__ballot_sync(kFull, aT) & lead);
            itertau += aT;
            // residual norms and the Newton correction are compared as squares (no square roots
            // on the iteration's critical path): resn2 = |res|^2, and the loop runs while
            // |dsg|^2 > (erroral |sg_in|)^2
            int iterNR = 0;
            double resoldn2 = 1.0;
            bool more = true;
            const double errlim2 = (p.erroral * sgnorm) * (p.erroral * sgnorm);
            bool aN = aT;
            while (true) {
                aN = aN && iterNR < 100 && more;
                if (!__any_sync(kFull, aN)) break;
                if (stats) {
                    c_nr += __popc(__ballot_sync(kFull, aN) & lead);
                    c_npass++;
                }
                iterNR += aN;
                int icut = 0;
                double resn2 = 4.0 * resoldn2, rho_c = 0.0;
                bool aC = aN;
                while (true) {
                    aC = aC && resn2 > resoldn2 && icut < 10;
                    if (!__any_sync(kFull, aC)) break;
                    if (stats) {
                        c_eval += __popc(__ballot_sync(kFull, aC) & lead);
                        c_pass++;
                    }
                    // plastic_strain_rate at sg (own systems)
                    double sgf[6];
                    xgather(X, sg_r, sgf);
                    double ep[5] = {0, 0, 0, 0, 0}, gdn[SPL], rsn[SPL];
#pragma unroll
                    for (int k = 0; k < SPL; k++) {
                        gdn[k] = 0.0;
                        rsn[k] = 0.0;
                        if (r + 6 * k < nsyst) {
                            double sc[5];
#pragma unroll
                            for (int c = 0; c < 5; c++) sc[c] = schm[(5 * k + c) * kXStride];
                            double rss = sc[0] * sgf[0] + sc[1] * sgf[1] + sc[2] * sgf[2] + sc[3] * sgf[3] + sc[4] * sgf[4];
                            // one reciprocal of the resistance for both quotients (rounding only:
                            // measured 2.5 % less time per launch, the same iteration counts)
                            const double tau = (rss - 0.0 < 0.0) ? TT[2 * k + 1] : TT[2 * k];
                            const double itau = 1.0 / tau;
                            rss = (rss - 0.0) * itau;
                            const double nk = ph.nrs[r + 6 * k];
                            const double dum = ph.gamd0[r + 6 * k] * powabs(rss, nk - 1.0, int_exp);
                            rsn[k] = nk * dum * itau;
                            gdn[k] = rss * dum;
#pragma unroll
                            for (int c = 0; c < 5; c++) ep[c] += sc[c] * gdn[k];
                        }
                    }
                    // component r of edotp: row r summed over the group in lane order
                    __syncwarp();
#pragma unroll
                    for (int c = 0; c < 5; c++) X.P[c * kXStride + lane] = ep[c];
                    __syncwarp();
                    double epr = 0.0;
                    if (r < 5) {
                        const double* e = X.P + r * kXStride + base;
                        epr = ((((e[0] + e[1]) + e[2]) + e[3]) + e[4]) + e[5];
                    }
                    double rho = epr - qp_r;
#pragma unroll
                    for (int j = 0; j < 6; j++) rho += Hrow[j] * sgf[j];
                    double rhof[6];
                    xgather(X, rho, rhof);
                    double rn = 0.0;
#pragma unroll
                    for (int j = 0; j < 6; j++) rn += Crow[j] * rhof[j];
                    const double rnn2 = xsum(X, rn * rn);
                    if (aC) {
#pragma unroll
                        for (int k = 0; k < SPL; k++) {
                            GD[k] = gdn[k];
                            RS[k] = rsn[k];
                        }
                        EPM[0] = epr;
                        SEV[0] = sg_r;
                        rho_c = rho;
                        resn2 = rnn2;
                        if (iterNR == 1) resoldn2 = resn2;
                        if (resn2 > resoldn2) sg_r = sgold_r + (sg_r - sgold_r) * 0.5;
                        icut++;
                    }
                }
                if (aN) {
                    resoldn2 = resn2;
                    sgold_r = sg_r;
                }
                // d(edotp)/d(sigma), packed upper triangle, partial over this lane's systems
                __syncwarp();
                {
                    double sc[SPL][5];
#pragma unroll
                    for (int k = 0; k < SPL; k++)
#pragma unroll
                        for (int c = 0; c < 5; c++) sc[k][c] = schm[(5 * k + c) * kXStride];
                    int q = 0;
#pragma unroll
                    for (int jj = 0; jj < 5; jj++)
#pragma unroll
                        for (int ii = 0; ii <= jj; ii++) {
                            double x = 0.0;
#pragma unroll
                            for (int k = 0; k < SPL; k++)
                                if (r + 6 * k < nsyst) x += sc[k][ii] * sc[k][jj] * RS[k];
                            X.P[q * kXStride + lane] = x;
                            q++;
                        }
                }
                __syncwarp();
                // row r of H = H0 + dd (dd summed over the group in lane order)
                double Hr[6];
#pragma unroll
                for (int j = 0; j < 6; j++) {
                    double x = 0.0;
                    if (j < 5 && r < 5) {
                        const int q = (r < j) ? j * (j + 1) / 2 + r : r * (r + 1) / 2 + j;  // dd(r, j), packed
                        const double* e = X.P + q * kXStride + base;
                        x = ((((e[0] + e[1]) + e[2]) + e[3]) + e[4]) + e[5];
                    }
                    Hr[j] = Hrow[j] + x;
                }
                // Gauss-Jordan elimination in the fixed order 0..5 (H is positive definite)
                double b = rho_c;
                bool sing = false;
#pragma unroll
                for (int k = 0; k < 6; k++) {
                    double pk[6];
#pragma unroll
                    for (int j = k; j < 6; j++) pk[j] = __shfl_sync(kFull, Hr[j], base + k);
                    const double bk = __shfl_sync(kFull, b, base + k);
                    sing = sing || (pk[k] == 0.0);
                    if (r != k) {
                        const double l = Hr[k] / pk[k];
#pragma unroll
                        for (int j = k + 1; j < 6; j++) Hr[j] -= l * pk[j];
                        b -= l * bk;
                    }
                }
                const double sg_new = sg_r - b / sel6(Hr, r);
                const double dsgnr = xsum(X, (sg_new - sgold_r) * (sg_new - sgold_r));
                if (aN) {
                    if (sing && r == 0) set_err(d.err, 1);
                    sg_r = sg_new;
                    more = sgnorm > 0.0 ? dsgnr > errlim2 : dsgnr > 0.0;
                }
            }
            if (p.iuphard) {  // harden (various_functions.f90:1439-1491)
                // the committed resistances and accumulated shear, loaded first so that their latency
                // overlaps the group sums and the exchange below
                const double gamma0 = d.gacumgr[v];
                double cr[SPL][2];
#pragma unroll
                for (int k = 0; k < SPL; k++) {
                    const int s = r + 6 * k;
                    cr[k][0] = s < nsyst ? d.crss[(2 * s) * N + v] : 0.0;
                    cr[k][1] = s < nsyst ? d.crss[(2 * s + 1) * N + v] : 0.0;
                }
                double dg = 0.0;
#pragma unroll
                for (int k = 0; k < SPL; k++)
                    if (r + 6 * k < nsyst) dg += fabs(GD[k]) * p.tdot;
                const double deltgam = xsum(X, dg);
                const double gamma1 = gamma0 + deltgam;
                // |slip rate| of the group's system 6k + q in exchange row k, column base + q
                __syncwarp();
#pragma unroll
                for (int k = 0; k < SPL; k++) X.P[k * kXStride + lane] = fabs(GD[k]);
                __syncwarp();
                double e2 = 0.0, tn[SPL][2];
                int vmode = -1;  // mode whose Voce increment is in voce (systems of one mode share it)
                double voce = 0.0;
#pragma unroll
                for (int k = 0; k < SPL; k++) {
                    const int s = r + 6 * k;
                    tn[k][0] = 0.0;  // systems beyond the phase's own get zero resistance, as harden leaves them
                    tn[k][1] = 0.0;
                    if (s < nsyst) {
                        int mode = 0, last = ph.nsm[0];
                        while (mode + 1 < ph.nmodes && s >= last) {
                            mode++;
                            last += ph.nsm[mode];
                        }
                        if (mode != vmode) {
                            const double tau1 = ph.tau1[mode], thet0 = ph.thet0[mode], thet1 = ph.thet1[mode];
                            const double fact = fabs(thet0 / tau1);
                            const double exp0 = exp(-fact * gamma0), exp1 = exp(-fact * gamma1);
                            voce = deltgam * thet1 + tau1 * (exp0 - exp1) + thet1 * (gamma0 * exp0 - gamma1 * exp1);
                            vmode = mode;
                        }
                        double dtau = 0.0;
#pragma unroll
                        for (int js = 0; js < 6 * SPL; js++)
                            if (js < nsyst) dtau = dtau + ph.hard[s * MS + js] * X.P[(js / 6) * kXStride + base + js % 6];
                        tn[k][0] = cr[k][0] + dtau * voce * p.tdot / deltgam;
                        tn[k][1] = cr[k][1] + dtau * voce * p.tdot / deltgam;
                    }
                    const double d0 = TT[2 * k] - tn[k][0], d1 = TT[2 * k + 1] - tn[k][1];
                    e2 += d0 * d0 + d1 * d1;
                }
                const double et = sqrt(xsum(X, e2)) / taun;
                if (aT) {
#pragma unroll
                    for (int k = 0; k < SPL; k++) {
                        TT[2 * k] = tn[k][0];
                        TT[2 * k + 1] = tn[k][1];
                    }
                    errtau = et;
                }
            } else if (aT) {
                errtau = 0.0;
            }
        }
        // |sg - lam|^2 at the final stress; |edot - D|^2 at the last evaluation, with
        // edot = edotp + S (sg - sgt) / dt + eth as elastic_strain_rate forms it
        double sgf[6], epf[6], ee = 0.0;
        {
            double srow[6], dsf[6];  // row r of S loaded before the exchange, to overlap its latency
#pragma unroll
            for (int j = 0; j < 6; j++) srow[j] = d.sg66[(6 * r + j) * N + v];
            xgather(X, (SEV[0] - sgt_r) / p.tdot, dsf);
#pragma unroll
            for (int j = 0; j < 6; j++) ee += srow[j] * dsf[j];
        }
        double edot_r = EPM[0] + ee;
        if (p.thermo) edot_r = edot_r + eth_r;
        const double dl = sg_r - LAM[0], de = edot_r - D_r;
        const double dsgnorm = xsum(X, dl * dl), ddgnorm = xsum(X, de * de);
        // outputs: sigma and edotp in the symmetric 3x3 form, slip rates and resistances
        xgather(X, sg_r, sgf);
        xgather(X, EPM[0], epf);
        epf[5] = 0.0;
        if (act) {
            double s6v[6], e6v[6];
            b6_to_s6(sgf, s6v);
            b6_to_s6(epf, e6v);
            d.sg[r * N + v] = sel6(s6v, r);
            d.edotp[r * N + v] = sel6(e6v, r);
#pragma unroll
            for (int k = 0; k < SPL; k++) {
                const int s = r + 6 * k;
                if (s < d.nsys) {
                    d.gamdot[s * N + v] = (s < nsyst) ? GD[k] : 0.0;
                    d.trialtau[(2 * s) * N + v] = TT[2 * k];
                    d.trialtau[(2 * s + 1) * N + v] = TT[2 * k + 1];
                }
            }
            if (r == 0) {
                const double w = d.wgtc[v];
                if (!(dsgnorm == dsgnorm) || !(ddgnorm == ddgnorm)) set_err(d.err, 2);
                accg[0] += dsgnorm * w;
                accg[1] += ddgnorm * w;
#pragma unroll
                for (int c = 0; c < 6; c++) {
                    accg[2 + c] += w * s6v[c];
                    accg[8 + c] += s6v[c] * w;
                }
            }
        }
        __syncwarp();  // every lane of a gas voxel's group has read sg before the update below writes it
        if (gas && r == 0) {  // dummy gas voxel: closed-form update by one lane
            const double w = d.wgtc[v];
            double lam[6], sgt6[6], D6[6], t[6], res[6], out[6], s6v[6], a[6], vg[9], vs[9];
            ld6(d.sg, N, v, a);
            s6_to_b6(a, lam);
            ld6(d.sgt, N, v, a);
            s6_to_b6(a, sgt6);
            ld9(d.velgrad, N, v, vg);
            sym33(vg, vs);
            t2_to_b6(vs, D6);
#pragma unroll
            for (int i = 0; i < 6; i++) t[i] = D6[i] + sgt6[i] / p.tdot * p.complgas;
#pragma unroll
            for (int i = 0; i < 6; i++) {
                double x = 0.0;
#pragma unroll
                for (int j = 0; j < 6; j++) x += d.c066mod[(6 * i + j) * N + v] * t[j];
                res[i] = lam[i] + x;
            }
#pragma unroll
            for (int i = 0; i < 6; i++) {
                double x = 0.0;
#pragma unroll
                for (int j = 0; j < 6; j++) x += d.cgas[(6 * i + j) * N + v] * res[j];
                out[i] = x;
            }
            b6_to_s6(out, s6v);
            st6(d.sg, N, v, s6v);
#pragma unroll
            for (int c = 0; c < 6; c++) d.edotp[c * N + v] = 0.0;
            for (int q = 0; q < d.nsys; q++) d.gamdot[q * N + v] = 0.0;
#pragma unroll
            for (int c = 0; c < 6; c++) accg[8 + c] += s6v[c] * w;
        }
    }
    __syncwarp();
    if (stats && lane == 0) {
        atomicAdd(d.nstats + 0, c_pass);
        atomicAdd(d.nstats + 1, c_eval);
        atomicAdd(d.nstats + 2, c_nr);
        atomicAdd(d.nstats + 3, c_tau);
        atomicAdd(d.nstats + 4, c_vox);
        atomicAdd(d.nstats + 5, c_npass);
    }
    double acc[14];
#pragma unroll
    for (int c = 0; c < 14; c++) acc[c] = lane < 5 ? accw[lane * 14 + c] : 0.0;
    reduce_store<14, 0>(acc, nullptr, d.partials, d.red + OFF_NEWTON, d.counters + CNT_NEWTON, vb);
}

template <int SPL>
__global__ void __launch_bounds__(256, 2) k_newton6p(Dev d, NewtonParams p) { body_newton6p<SPL>(d, p, hw_vb()); }

// The local-solve kernel of a solve: 0 k_newton6p<2>, 1 k_newton6p<4> (symmetric form, no modAL,
// at most kMaxPhaseSmem phases), 2/3 k_newton6<2/4, modal>, 4/5 k_newton6<2/4, no modAL>, and
// 6/7 the one-thread-per-voxel kernel k_newton<12/24> (EVP_NEWTON_ONE_THREAD=1, kept for comparison).
static int newton_variant(const Dev& d, int modal) {
    static const bool one_thread = [] {
        const char* e = getenv("EVP_NEWTON_ONE_THREAD");
        return e && e[0] == '1';
    }();
    const bool big = d.nsys > 12;
    if (one_thread) return big ? 7 : 6;
    if (!modal && d.nph <= kMaxPhaseSmem) return big ? 1 : 0;
    if (modal) return big ? 3 : 2;
    return big ? 5 : 4;
}
static int newton_grid(const Dev& d, int variant) {
    if (variant >= 6) {
        const long long g = (d.N + kNewtonBlock - 1) / kNewtonBlock;
        return (int)(g < 148LL * 16 ? g : 148LL * 16);
    }
    // one wave: the two blocks of 256 that fit each of the 148 SMs, every warp taking every
    // (blocks x 8)-th batch of five voxels (measured on 64^3: 0.685 ms per launch against 0.766
    // with 24 blocks per SM, where every block staged the phases, waited at its end for its
    // slowest warp and folded its own sums)
    const long long warps = (d.N + 4) / 5;
    const long long g = (warps + 7) / 8;  // 8 warps per block of 256
    return (int)(g < 148LL * 2 ? g : 148LL * 2);
}
static size_t newton_smem(const Dev& d, int variant) {
    switch (variant) {
        case 0: return newton6p_smem_bytes(2, d.nph);
        case 1: return newton6p_smem_bytes(4, d.nph);
        case 2: case 4: return newton6_smem_bytes(2);
        case 3: case 5: return newton6_smem_bytes(4);
        default: return 0;
    }
}
template <int V>
__global__ void __launch_bounds__(V >= 6 ? 128 : 256, 2) kb_newton(const __grid_constant__ BatchParams P);
static void newton_configure() {
    static std::once_flag once;
    std::call_once(once, [] {
        const int lim = 200 * 1024;
        cudaFuncSetAttribute(k_newton6p<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
        cudaFuncSetAttribute(k_newton6p<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
        cudaFuncSetAttribute(k_newton6<2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
        cudaFuncSetAttribute(k_newton6<2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
        cudaFuncSetAttribute(kb_newton<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
        cudaFuncSetAttribute(kb_newton<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
        cudaFuncSetAttribute(kb_newton<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
        cudaFuncSetAttribute(kb_newton<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
        cudaFuncSetAttribute(kb_newton<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
        cudaFuncSetAttribute(kb_newton<5>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    });
}

void launch_newton(const Dev& d, const NewtonParams& p, cudaStream_t st) {
    newton_configure();
    const int v = newton_variant(d, p.modal);
    const int grid = newton_grid(d, v);
    const size_t sm = newton_smem(d, v);
    switch (v) {
        case 0: k_newton6p<2><<<grid, 256, sm, st>>>(d, p); break;
        case 1: k_newton6p<4><<<grid, 256, sm, st>>>(d, p); break;
        case 2: k_newton6<2, true><<<grid, 256, sm, st>>>(d, p); break;
        case 3: k_newton6<4, true><<<grid, 256, sm, st>>>(d, p); break;
        case 4: k_newton6<2, false><<<grid, 256, sm, st>>>(d, p); break;
        case 5: k_newton6<4, false><<<grid, 256, sm, st>>>(d, p); break;
        case 6: k_newton<12><<<grid, kNewtonBlock, 0, st>>>(d, p); break;
        default: k_newton<24><<<grid, kNewtonBlock, 0, st>>>(d, p); break;
    }
}

// ---------------------------------------------------------------- batched launches of the iteration's voxel passes
// Each block finds its member in the launch's parameter (binary search on blk0), reads
// the member's control block and runs the same body as the member's single-solve
// launch, on the member's own block coordinates.  Blocks of members that are not
// iterating (converged, waiting for the host) exit at once.
template <bool GAS>
__global__ void __launch_bounds__(kBlock, 2) kb_corr(const __grid_constant__ BatchParams P) {
    __shared__ CorrParams p;
    __shared__ int go;
    const Job& jb = batch_job(P);
    const BatchSolve& m = P.E[jb.solve];
    if (threadIdx.x == 0) {
        go = m.ctl->active;
        p = m.ctl->corr;
    }
    __syncthreads();
    if (!go) return;
    body_corr<GAS>(m.d, p, job_vb(jb));
}
template <int V>
__global__ void __launch_bounds__(V >= 6 ? 128 : 256, 2) kb_newton(const __grid_constant__ BatchParams P) {
    __shared__ NewtonParams ps;
    __shared__ int go;
    const Job& jb = batch_job(P);
    const BatchSolve& m = P.E[jb.solve];
    if (threadIdx.x == 0) {
        go = m.ctl->active;
        ps = m.ctl->newton;
    }
    __syncthreads();
    if (!go) return;
    const NewtonParams p = ps;  // in registers, as a single-solve launch's parameter
    const VB vb = job_vb(jb);
    if constexpr (V == 0) body_newton6p<2>(m.d, p, vb);
    else if constexpr (V == 1) body_newton6p<4>(m.d, p, vb);
    else if constexpr (V == 2) body_newton6<2, true>(m.d, p, vb);
    else if constexpr (V == 3) body_newton6<4, true>(m.d, p, vb);
    else if constexpr (V == 4) body_newton6<2, false>(m.d, p, vb);
    else if constexpr (V == 5) body_newton6<4, false>(m.d, p, vb);
    else if constexpr (V == 6) body_newton1<12>(m.d, p, vb);
    else body_newton1<24>(m.d, p, vb);
}

void member_jobs_voxel(const Dev& d, int modal, MemberJobs& mj) {
    newton_configure();
    auto one_d = [&](int k, int grid, int thr, size_t sm, int variant) {
        mj.job[0][k] = Job{0, 0, grid, 1, 1, 0};
        mj.threads[0][k] = thr;
        mj.smem[0][k] = sm;
        mj.variant[0][k] = variant;
    };
    one_d(BK_CORR, d.grid < 148 * 2 ? d.grid : 148 * 2, kBlock, 0, d.cgas ? 0 : 1);
    const int v = newton_variant(d, modal);
    one_d(BK_NEWTON, newton_grid(d, v), v >= 6 ? kNewtonBlock : 256, newton_smem(d, v), v);
}

void launch_batched_voxel(const BatchLaunch& L, const BatchParams& P, cudaStream_t st) {
    switch (L.kind) {
        case BK_CORR:
            if (L.variant == 0) kb_corr<true><<<L.blocks, L.threads, 0, st>>>(P);
            else kb_corr<false><<<L.blocks, L.threads, 0, st>>>(P);
            break;
        case BK_NEWTON:
            switch (L.variant) {
                case 0: kb_newton<0><<<L.blocks, L.threads, L.smem, st>>>(P); break;
                case 1: kb_newton<1><<<L.blocks, L.threads, L.smem, st>>>(P); break;
                case 2: kb_newton<2><<<L.blocks, L.threads, L.smem, st>>>(P); break;
                case 3: kb_newton<3><<<L.blocks, L.threads, L.smem, st>>>(P); break;
                case 4: kb_newton<4><<<L.blocks, L.threads, L.smem, st>>>(P); break;
                case 5: kb_newton<5><<<L.blocks, L.threads, L.smem, st>>>(P); break;
                case 6: kb_newton<6><<<L.blocks, L.threads, L.smem, st>>>(P); break;
                default: kb_newton<7><<<L.blocks, L.threads, L.smem, st>>>(P); break;
            }
            break;
        default: break;
    }
}

// ---------------------------------------------------------------- k_upd1
template <int NS>
__global__ void __launch_bounds__(kBlock) k_upd1(Dev d, Upd1Params p) {
    const long long N = d.N;
    double s[39], mx[1] = {0.0};
#pragma unroll
    for (int c = 0; c < 39; c++) s[c] = 0.0;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < N; v += (long long)gridDim.x * blockDim.x) {
        const bool gas = d.gas[v];
        // accepted-step commit (LS-EVPFFT.f90:432-446)
        double e6[6], a6[6], vg[9], vs[9];
        ld6(d.edotp, N, v, e6);
        ld6(d.ept, N, v, a6);
#pragma unroll
        for (int c = 0; c < 6; c++) a6[c] = a6[c] + e6[c] * p.tdot;
        st6(d.ept, N, v, a6);
        ld6(d.sg, N, v, a6);
        st6(d.sgt, N, v, a6);
        ld9(d.velgrad, N, v, vg);
        sym33(vg, vs);
        ld6(d.disgradsym, N, v, a6);
        double vs6[6];
        t2_to_s6(vs, vs6);
#pragma unroll
        for (int c = 0; c < 6; c++) a6[c] = a6[c] + vs6[c] * p.tdot;
        st6(d.disgradsym, N, v, a6);
        double e9[9];
        s6_to_t2(e6, e9);
        d.epvm[v] = d.epvm[v] + vm_strain(e9) * p.tdot;
        const double evm = vm_strain(vs);
        if (!gas) mx[0] = fmax(mx[0], evm);
        if (!p.iupdate) continue;
        if (!gas) {  // update_plastic_defgrad (various_functions.f90:1748-1827)
            const PhaseDev& ph = d.ph[d.phase[v]];
            double ag[9], Lp[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            ld9(d.ag, N, v, ag);
            for (int is = 0; is < ph.nsyst; is++) {
                double dn[3], db[3];
                for (int i = 0; i < 3; i++) {
                    dn[i] = ag[3 * i] * ph.dnca[3 * is] + ag[3 * i + 1] * ph.dnca[3 * is + 1] + ag[3 * i + 2] * ph.dnca[3 * is + 2];
                    db[i] = ag[3 * i] * ph.dbca[3 * is] + ag[3 * i + 1] * ph.dbca[3 * is + 1] + ag[3 * i + 2] * ph.dbca[3 * is + 2];
                }
                const double gd = d.gamdot[is * N + v];
                for (int i = 0; i < 3; i++)
                    for (int j = 0; j < 3; j++) Lp[3 * i + j] = Lp[3 * i + j] + db[i] * dn[j] * gd;
            }
            double dl[9], ex[9], fp[9];
            for (int c = 0; c < 9; c++) dl[c] = Lp[c] * p.tdot;
            if (expm_adaptive(dl, ex) != 0) set_err(d.err, 1);
            ld9(d.Fp, N, v, fp);
            mm3(ex, fp, fp);
            st9(d.Fp, N, v, fp);
        }
        // update_defgrad (various_functions.f90:2152-2282)
        double dl[9], ex[9], F[9], Fi[9];
        for (int c = 0; c < 9; c++) dl[c] = vg[c] * p.tdot;
        if (expm_adaptive(dl, ex) != 0) set_err(d.err, 1);
        ld9(d.F, N, v, F);
        mm3(ex, F, F);
        const double detF = det33(F);
        if (inv3u(F, Fi) != 0) set_err(d.err, 1);
        st9(d.F, N, v, F);
        st9(d.Finv, N, v, Fi);
        st9(d.Finc, N, v, ex);
        d.detF[v] = detF;
        d.wgtc[v] = d.wgt * detF;
#pragma unroll
        for (int c = 0; c < 9; c++) {
            s[c] += F[c] * d.wgt;
            s[9 + c] += Fi[c] * d.wgt * detF;
            if (gas) s[27 + c] += Fi[c] * d.wgt * detF;
            else s[18 + c] += Fi[c] * d.wgt * detF;
        }
        if (gas) s[37] += d.wgt * detF;
        else s[36] += d.wgt * detF;
        s[38] += detF * d.wgt;
    }
    reduce_store<39, 1>(s, mx, d.partials, d.red + OFF_UPD1, d.counters + CNT_UPD1, hw_vb());
}
void launch_upd1(const Dev& d, const Upd1Params& p, cudaStream_t st) {
    if (d.nsys <= 12) k_upd1<12><<<d.grid, kBlock, 0, st>>>(d, p);
    else k_upd1<24><<<d.grid, kBlock, 0, st>>>(d, p);
}

// ---------------------------------------------------------------- k_upd2
__global__ void __launch_bounds__(kBlock) k_upd2(Dev d, Upd2Params p) {
    const long long N = d.N;
    const double dav = __ldcg(&d.red[OFF_UPD1 + 38]);
    double s[9];
#pragma unroll
    for (int c = 0; c < 9; c++) s[c] = 0.0;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < N; v += (long long)gridDim.x * blockDim.x) {
        const bool gas = d.gas[v];
        const double w = d.wgtc[v] / dav;
        d.wgtc[v] = w;
        double Finc[9], Feinc[9];
        ld9(d.Finc, N, v, Finc);
        if (!gas) {
            // update_elstic_defgrad (various_functions.f90:2285-2324): Fe = F (Fp Fini)^-1, Fini = I
            // unless an initial displacement field was given
            const PhaseDev& ph = d.ph[d.phase[v]];
            double Fe[9], Feo[9], Fp[9], Fpi[9], F[9];
            ld9(d.Fe, N, v, Fe);
            if (inv3u(Fe, Feo) != 0) set_err(d.err, 1);
            ld9(d.Fp, N, v, Fp);
            if (d.Fini) {
                double Fi0[9], FpFi[9];
                ld9(d.Fini, N, v, Fi0);
                mm3(Fp, Fi0, FpFi);
                if (inv3u(FpFi, Fpi) != 0) set_err(d.err, 1);
            } else if (inv3u(Fp, Fpi) != 0) {
                set_err(d.err, 1);
            }
            ld9(d.F, N, v, F);
            mm3(F, Fpi, Fe);
            mm3(Fe, Feo, Feinc);
            st9(d.Fe, N, v, Fe);
            st9(d.Feinc, N, v, Feinc);
            // update_el_stiff (various_functions.f90:2327-2402)
            // (the rotation of the crystal stiffness by aa = Fe ag as two 6x6 products in the
            // b-basis, Q c Q^T with Q = rot_b66(aa), instead of index by index over 3x3x3x3 and
            // chg_basis: the same tensor, rounding apart)
            double ag[9], aa[9], Q[36], cc[36], c66[36];
            ld9(d.ag, N, v, ag);
            mm3(Fe, ag, aa);
            const double detFe = det33(Fe);
            rot_b66(aa, Q);
            t4_to_b66(ph.C, cc);
            congruence6(Q, cc, 1.0 / detFe, c66);
            if (inv_unrolled<6>(c66) != 0) set_err(d.err, 1);
#pragma unroll
            for (int c = 0; c < 36; c++) d.sg66[c * N + v] = c66[c];
        } else {
            ld9(d.Feinc, N, v, Feinc);
        }
        // update_tensor_config pass 1 (various_functions.f90:2425-2466)
        const double detei = det33(Feinc);
        double Fii[9];
        if (inv3u(Finc, Fii) != 0) set_err(d.err, 1);
        if (!gas) {
            double R[9], U[9], t[9], m[9], a6[6];
            polar(Finc, R, U);
            ld6(d.disgradsym, N, v, a6);
            s6_to_t2(a6, m);
            mm3(R, m, t);
            mm3_bt(t, R, m);
            t2_to_s6(m, a6);
            st6(d.disgradsym, N, v, a6);
            ld6(d.ept, N, v, a6);
            s6_to_t2(a6, m);
            mm3(R, m, t);
            mm3_bt(t, R, m);
            t2_to_s6(m, a6);
            st6(d.ept, N, v, a6);
            ld6(d.sgt, N, v, a6);
            s6_to_t2(a6, m);
            mm3(Feinc, m, t);
            mm3_bt(t, Feinc, m);
            for (int c = 0; c < 9; c++) m[c] = m[c] / detei;
            t2_to_s6(m, a6);
            st6(d.sgt, N, v, a6);
        }
        double vg[9];
        ld9(d.velgrad, N, v, vg);
        mm3(vg, Fii, vg);
        st9(d.velgrad, N, v, vg);
#pragma unroll
        for (int c = 0; c < 9; c++) s[c] += vg[c] * w;
    }
    // reduce; the last block forms du2 = (<L>_prev - <L>) inv(<F^{-1}>_c)
    __shared__ double sh[9][32];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int f = 0; f < 9; f++) {
        double x = s[f];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) sh[f][warp] = x;
    }
    __syncthreads();
    if (warp == 0) {
        for (int f = 0; f < 9; f++) {
            double x = lane < nw ? sh[f][lane] : 0.0;
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            if (lane == 0) d.partials[(size_t)f * gridDim.x + blockIdx.x] = x;
        }
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = (atomicAdd(d.counters + CNT_UPD2, 1u) == gridDim.x - 1);
    __syncthreads();
    __shared__ double fsum[9];
    if (last) {
        __threadfence();
        for (int f = warp; f < 9; f += nw) {
            const double x = fold_sum(d.partials, gridDim.x, f, lane);
            if (lane == 0) fsum[f] = x;
        }
        __syncthreads();
    }
    if (last && threadIdx.x == 0) {
        double va[9], fc[9], di[9], dd[9], du[9];
        for (int f = 0; f < 9; f++) {
            va[f] = fsum[f];
            fc[f] = __ldcg(&d.red[OFF_UPD1 + 9 + f]) / dav;
        }
        if (inv3u(fc, di) != 0) set_err(d.err, 1);
        for (int f = 0; f < 9; f++) dd[f] = p.velgradavg[f] - va[f];
        mm3(dd, di, du);
        for (int f = 0; f < 9; f++) d.red[OFF_DU2 + f] = du[f];
        d.counters[CNT_UPD2] = 0;
    }
}
void launch_upd2(const Dev& d, const Upd2Params& p, cudaStream_t st) { k_upd2<<<d.grid, kBlock, 0, st>>>(d, p); }

// ---------------------------------------------------------------- k_upd3
template <int NS>
__global__ void __launch_bounds__(kBlock, 2) k_upd3(Dev d, Upd3Params p) {
    const long long N = d.N;
    __shared__ double du[9];
    if (threadIdx.x < 9) du[threadIdx.x] = p.iupdate ? __ldcg(&d.red[OFF_DU2 + threadIdx.x]) : 0.0;
    __syncthreads();
    double s[30];
#pragma unroll
    for (int c = 0; c < 30; c++) s[c] = 0.0;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < N; v += (long long)gridDim.x * blockDim.x) {
        const bool gas = d.gas[v];
        if (p.iupdate) {
            double fi[9], t[9], vg[9];
            ld9(d.Finv, N, v, fi);
            mm3(du, fi, t);
            ld9(d.velgrad, N, v, vg);
#pragma unroll
            for (int c = 0; c < 9; c++) vg[c] = vg[c] + t[c];
            st9(d.velgrad, N, v, vg);
        }
        if (gas) continue;
        const PhaseDev& ph = d.ph[d.phase[v]];
        double gd[NS];
#pragma unroll
        for (int q = 0; q < NS; q++) gd[q] = (q < d.nsys) ? d.gamdot[q * N + v] : 0.0;
        if (p.iuphard) {  // update_hardening (various_functions.f90:1493-1523)
            double tn[NS][2], g1;
            harden<NS>(ph, d.crss, N, v, gd, d.gacumgr[v], p.tdot, tn, g1);
#pragma unroll
            for (int q = 0; q < NS; q++)
                if (q < d.nsys) {
                    d.crss[(2 * q) * N + v] = tn[q][0];
                    d.crss[(2 * q + 1) * N + v] = tn[q][1];
                    d.trialtau[(2 * q) * N + v] = tn[q][0];
                    d.trialtau[(2 * q + 1) * N + v] = tn[q][1];
                }
            d.gacumgr[v] = g1;
        }
        const double w = d.wgtc[v];
        double a[6];
        ld6(d.ept, N, v, a);
#pragma unroll
        for (int c = 0; c < 6; c++) s[c] += a[c] * w;
        if (v == p.vlast) {
            for (int c = 0; c < 6; c++) d.red[OFF_UPD3 + 36 + c] = a[c];
        }
        ld6(d.disgradsym, N, v, a);
#pragma unroll
        for (int c = 0; c < 6; c++) s[6 + c] += a[c] * w;
        if (v == p.vlast) {
            for (int c = 0; c < 6; c++) d.red[OFF_UPD3 + 30 + c] = a[c];
            d.red[OFF_UPD3 + 42] = w;
        }
        ld6(d.edotp, N, v, a);
#pragma unroll
        for (int c = 0; c < 6; c++) s[12 + c] += a[c] * w;
        ld6(d.sgt, N, v, a);
#pragma unroll
        for (int c = 0; c < 6; c++) s[18 + c] += a[c] * w;
        s[24] += d.gacumgr[v];
        s[25] += 1.0;
#pragma unroll
        for (int q = 0; q < NS; q++)
            if (q < ph.nsyst) {
                const double gs = 0.5 * (d.crss[(2 * q) * N + v] + d.crss[(2 * q + 1) * N + v]);
                s[26] += gs;
                s[27] += 1.0;
                s[28] += fabs(gd[q]);
                s[29] += fabs(gd[q]) * gs;
            }
    }
    reduce_store<30, 0>(s, nullptr, d.partials, d.red + OFF_UPD3, d.counters + CNT_UPD3, hw_vb());
}
void launch_upd3(const Dev& d, const Upd3Params& p, cudaStream_t st) {
    if (d.nsys <= 12) k_upd3<12><<<d.grid, kBlock, 0, st>>>(d, p);
    else k_upd3<24><<<d.grid, kBlock, 0, st>>>(d, p);
}

// ---------------------------------------------------------------- k_diag
// sums: s2a swa s2s sws s2g swg | maxes: mxa mxs mxg vms vmg rms rmg sms smg ccs ccg cgg
// min detF (all), and (min, last index) for solid and gas voxels.
struct MinIdx {
    double v;
    long long i;
};
__device__ __forceinline__ MinIdx min_last(MinIdx a, MinIdx b) {
    if (b.v < a.v) return b;
    if (a.v < b.v) return a;
    return (b.i > a.i) ? b : a;
}
__global__ void __launch_bounds__(kBlock, 2) k_diag(Dev d, double Lfloor) {
    const long long N = d.N;
    double s[6] = {0, 0, 0, 0, 0, 0};
    double m[13];
#pragma unroll
    for (int c = 0; c < 12; c++) m[c] = 0.0;
    m[12] = -EVP_HUGE;  // max of -detF
    MinIdx ms = {EVP_HUGE, -1}, mg = {EVP_HUGE, -1};
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < N; v += (long long)gridDim.x * blockDim.x) {
        const bool gas = d.gas[v];
        double vg[9], vs[9], Fi[9];
        ld9(d.velgrad, N, v, vg);
        ld9(d.s_velgrad, N, v, vs);
        double dl = 0.0, l0 = 0.0;
#pragma unroll
        for (int c = 0; c < 9; c++) { dl += (vg[c] - vs[c]) * (vg[c] - vs[c]); l0 += vs[c] * vs[c]; }
        dl = sqrt(dl);
        l0 = sqrt(l0);
        const double rel = dl / fmax(l0, Lfloor);
        const double w = d.wgtc[v];
        s[0] += (rel * rel) * w; s[1] += w; m[0] = fmax(m[0], rel);
        const double detF = d.detF[v];
        m[12] = fmax(m[12], -detF);
        ld9(d.Finc, N, v, Fi);
        double vi, ro, st, Ji;
        stretch_rot(Fi, true, vi, ro, st, Ji);
        double c66[36];
        for (int c = 0; c < 36; c++) c66[c] = d.c066mod[c * N + v];
        const double cc = cond1_est_6x6(c66);
        if (gas) {
            MinIdx t = {detF, v};
            mg = min_last(mg, t);
            s[4] += (rel * rel) * w; s[5] += w; m[2] = fmax(m[2], rel);
            m[4] = fmax(m[4], vi); m[6] = fmax(m[6], ro); m[8] = fmax(m[8], st);
            m[10] = fmax(m[10], cc);
            for (int c = 0; c < 36; c++) c66[c] = d.cgas[c * N + v];
            m[11] = fmax(m[11], cond1_est_6x6(c66));
        } else {
            MinIdx t = {detF, v};
            ms = min_last(ms, t);
            s[2] += (rel * rel) * w; s[3] += w; m[1] = fmax(m[1], rel);
            m[3] = fmax(m[3], vi); m[5] = fmax(m[5], ro); m[7] = fmax(m[7], st);
            m[9] = fmax(m[9], cc);
        }
    }
    // (min, last index) pairs reduced first, by a fixed-order warp/block tree
    __shared__ MinIdx shm[2][32];
    __shared__ bool lastblk;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int o = 16; o > 0; o >>= 1) {
        MinIdx a = {__shfl_down_sync(0xffffffffu, ms.v, o), __shfl_down_sync(0xffffffffu, ms.i, o)};
        MinIdx b = {__shfl_down_sync(0xffffffffu, mg.v, o), __shfl_down_sync(0xffffffffu, mg.i, o)};
        ms = min_last(ms, a);
        mg = min_last(mg, b);
    }
    if (lane == 0) { shm[0][warp] = ms; shm[1][warp] = mg; }
    __syncthreads();
    MinIdx* pm = reinterpret_cast<MinIdx*>(d.partials + (size_t)gridDim.x * 19);
    if (threadIdx.x == 0) {
        MinIdx a = shm[0][0], b = shm[1][0];
        for (int q = 1; q < nw; q++) { a = min_last(a, shm[0][q]); b = min_last(b, shm[1][q]); }
        pm[2 * blockIdx.x] = a;
        pm[2 * blockIdx.x + 1] = b;
    }
    __syncthreads();
    reduce_store<6, 13>(s, m, d.partials, d.red + OFF_DIAG, d.counters + CNT_DIAG, hw_vb());
    // reduce_store reset the counter; use a second counter pass for the pairs
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) lastblk = (atomicAdd(d.counters + CNT_DIAG2, 1u) == gridDim.x - 1);
    __syncthreads();
    if (lastblk && threadIdx.x == 0) {
        __threadfence();
        MinIdx a = {EVP_HUGE, -1}, b = {EVP_HUGE, -1};
        unsigned q = 0;
        for (; q + 8 <= gridDim.x; q += 8) {  // eight blocks' pairs loaded at a time, folded in block order
            MinIdx x[8], y[8];
#pragma unroll
            for (int i = 0; i < 8; i++) {
                x[i] = MinIdx{__ldcg(&pm[2 * (q + i)].v), __ldcg(&pm[2 * (q + i)].i)};
                y[i] = MinIdx{__ldcg(&pm[2 * (q + i) + 1].v), __ldcg(&pm[2 * (q + i) + 1].i)};
            }
#pragma unroll
            for (int i = 0; i < 8; i++) {
                a = min_last(a, x[i]);
                b = min_last(b, y[i]);
            }
        }
        for (; q < gridDim.x; q++) {
            MinIdx x = {__ldcg(&pm[2 * q].v), __ldcg(&pm[2 * q].i)};
            MinIdx y = {__ldcg(&pm[2 * q + 1].v), __ldcg(&pm[2 * q + 1].i)};
            a = min_last(a, x);
            b = min_last(b, y);
        }
        d.red[OFF_DIAG + 19] = a.v;
        d.red[OFF_DIAG + 20] = (double)a.i;
        d.red[OFF_DIAG + 21] = b.v;
        d.red[OFF_DIAG + 22] = (double)b.i;
        d.counters[CNT_DIAG2] = 0;
    }
}
void launch_diag(const Dev& d, double Lfloor, cudaStream_t st) { k_diag<<<d.grid, kBlock, 0, st>>>(d, Lfloor); }

// ---------------------------------------------------------------- k_c0
template <int NS>
__global__ void __launch_bounds__(kC0Block) k_c0(Dev d, double tdot, double tdotref) {
    const long long N = d.N;
    // each thread's 72 running sums in its own shared-memory slice (registers hold the per-voxel work)
    extern __shared__ double c0acc[];
    double* const s = c0acc + threadIdx.x * 72;
    for (int c = 0; c < 72; c++) s[c] = 0.0;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < N; v += (long long)gridDim.x * blockDim.x) {
        if (d.gas[v]) continue;
        const PhaseDev& ph = d.ph[d.phase[v]];
        double a6[6], sg[6];
        ld6(d.sg, N, v, a6);
        s6_to_b6(a6, sg);
        double tt[NS][2], ep[6], dd[15], gd[NS];
#pragma unroll
        for (int q = 0; q < NS; q++) {
            tt[q][0] = (q < d.nsys) ? d.trialtau[(2 * q) * N + v] : 1.0;
            tt[q][1] = (q < d.nsys) ? d.trialtau[(2 * q + 1) * N + v] : 1.0;
        }
        constitutive<NS>(ph, d.sch, N, v, tt, sg, ep, dd, gd);
        double tr[36];
#pragma unroll
        for (int i = 0; i < 6; i++)
#pragma unroll
            for (int j = 0; j < 6; j++) tr[6 * i + j] = d.sg66[(6 * i + j) * N + v] / tdot * tdot / tdotref + dd_at(dd, i, j);
        if (inv_unrolled<6>(tr) != 0) set_err(d.err, 1);
        // dsg = tr in the b-basis (summed here, expanded to 3x3x3x3 on the host); the PK1 tangent
        // dpg_ijkl = J sum_mn dsg_imkn Fi_jm Fi_ln has the b-basis components J T(Fi) tr T(Fi)^T
        double Fi[9], T[36], dp6[36];
        ld9(d.Finv, N, v, Fi);
        const double detF = d.detF[v], w = d.wgtc[v];
        basis_T(Fi, T);
        congruence6(T, tr, detF, dp6);
#pragma unroll
        for (int c = 0; c < 36; c++) s[c] += tr[c] * w;
#pragma unroll
        for (int c = 0; c < 36; c++) s[36 + c] += dp6[c] * d.wgt;
    }
    reduce_store<72, 0>(s, nullptr, d.partials, d.red + OFF_C0, d.counters + CNT_C0, hw_vb());
}
void launch_c0(const Dev& d, double tdot, double tdotref, cudaStream_t st) {
    const size_t sm = (size_t)kC0Block * 72 * sizeof(double);
    // four blocks per SM (the 255-register bound allows four of 64 threads): one wave, each
    // thread several voxels, and a fold of 592 block partials per field instead of 2368
    // (measured 624 -> 498 us at 64^3)
    const long long g = (d.N + kC0Block - 1) / kC0Block;
    const int grid = (int)(g < 148LL * 4 ? g : 148LL * 4);
    if (d.nsys <= 12) {
        cudaFuncSetAttribute(k_c0<12>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        k_c0<12><<<grid, kC0Block, sm, st>>>(d, tdot, tdotref);
    } else {
        cudaFuncSetAttribute(k_c0<24>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        k_c0<24><<<grid, kC0Block, sm, st>>>(d, tdot, tdotref);
    }
}

// ---------------------------------------------------------------- k_kinematic
__global__ void __launch_bounds__(kBlock) k_kinematic(Dev d, double tdot_step) {
    const long long N = d.N;
    double m[4] = {0.0, 0.0, 0.0, -EVP_HUGE};
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < N; v += (long long)gridDim.x * blockDim.x) {
        double L[9], Fi[9];
        ld9(d.velgrad, N, v, L);
        for (int c = 0; c < 9; c++) L[c] = L[c] * tdot_step;
        if (expm_adaptive(L, Fi) != 0) set_err(d.err, 1);
        double vi, ro, st, Ji;
        stretch_rot(Fi, false, vi, ro, st, Ji);
        m[0] = fmax(m[0], vi);
        m[1] = fmax(m[1], ro);
        m[2] = fmax(m[2], st);
        m[3] = fmax(m[3], -(d.detF[v] * Ji));
    }
    reduce_store<0, 4>(nullptr, m, d.partials, d.red + OFF_KIN, d.counters + CNT_KIN, hw_vb());
}
void launch_kinematic(const Dev& d, double tdot_step, cudaStream_t st) { k_kinematic<<<d.grid, kBlock, 0, st>>>(d, tdot_step); }

// ---------------------------------------------------------------- k_cell2node
__global__ void __launch_bounds__(kBlock) k_cell2node(Dev d, double tdot, int ideriv) {
    const int n1 = d.n1, n2 = d.n2, n3 = d.n3;
    const long long nn1 = n1 + 1, nn2 = n2 + 1;
    const long long nnode = nn1 * nn2 * d.n3node;
    __shared__ double va[9];
    if (threadIdx.x < 9) va[threadIdx.x] = __ldcg(&d.red[OFF_DC + 2 * threadIdx.x]) * d.wgt;
    __syncthreads();
    const long long N = d.N;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nnode; q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q % nn1) + 1, j = (int)((q / nn1) % nn2) + 1, k = (int)(q / (nn1 * nn2)) + 1;
        double dn[3];
        if (ideriv != 2) {
            int k1 = k - 1, k2 = k, j1 = j - 1, j2 = j, i1 = i - 1, i2 = i;
            if (k1 == 0) k1 = n3;
            if (k2 == n3 + 1) k2 = 1;
            if (j1 == 0) j1 = n2;
            if (j2 == n2 + 1) j2 = 1;
            if (i1 == 0) i1 = n1;
            if (i2 == n1 + 1) i2 = 1;
            auto c = [&](int a, int b, int e, int l) {
                return d.dv3[l * N + (a - 1) + (long long)n1 * ((b - 1) + (long long)n2 * (e - 1))];
            };
            for (int l = 0; l < 3; l++)
                dn[l] = (c(i2, j2, k2, l) + c(i1, j2, k2, l) + c(i2, j1, k2, l) + c(i2, j2, k1, l) + c(i1, j1, k2, l) +
                         c(i1, j2, k1, l) + c(i2, j1, k1, l) + c(i1, j1, k1, l)) * 0.125;
        } else {
            long long vv = ((i - 1) % n1) + (long long)n1 * (((j - 1) % n2) + (long long)n2 * ((k - 1) % n3));
            for (int l = 0; l < 3; l++) dn[l] = d.dv3[l * N + vv];
        }
        const double x[3] = {(double)i - 0.5, (double)j - 0.5, (d.n3node == 1) ? 0.0 : (double)k - 0.5};
        for (int l = 0; l < 3; l++) {
            const double sv = va[3 * l] * x[0] + va[3 * l + 1] * x[1] + va[3 * l + 2] * x[2];
            d.xnode[3 * q + l] = d.xnode[3 * q + l] + (sv + dn[l]) * tdot;
        }
    }
}
void launch_cell2node(const Dev& d, double tdot, int ideriv, cudaStream_t st) {
    k_cell2node<<<d.grid, kBlock, 0, st>>>(d, tdot, ideriv);
}

// ---------------------------------------------------------------- k_goperr0
__device__ __forceinline__ void spatial_freq(int kx, int ky, int kz, int n1, int n2, int n3, double* xi) {
    const double twopi = 2.0 * EVP_PI;
    xi[0] = (kx + 1 <= n1 / 2) ? twopi * (double)kx / (double)n1 : twopi * (double)(kx - n1) / (double)n1;
    xi[1] = (ky + 1 <= n2 / 2) ? twopi * (double)ky / (double)n2 : twopi * (double)(ky - n2) / (double)n2;
    if (n3 == 1) xi[2] = 0.0;
    else xi[2] = (kz + 1 <= n3 / 2) ? twopi * (double)kz / (double)n3 : twopi * (double)(kz - n3) / (double)n3;
}
// Green operator at one frequency point, all three forms of form_G (various_functions.f90:640-785):
// IGAMMA 0 continuous (Nyquist planes: -s0), 1 discrete central differences followed by four
// projections g <- -g1 : c0 : g, 2 rotated scheme (zero where two Nyquist planes meet).
// kx, ky, kz are 0-based indices of the full spectrum.  Returns 1 for a singular acoustic tensor
// or a complex rotated-scheme D (the reference stops there).
__device__ int goper_at(int igamma, int kx, int ky, int kz, int n1, int n2, int n3, const double* c0, const double* s0,
                        double* g) {
    const bool nx = (n1 % 2 == 0 && kx == n1 / 2), ny = (n2 % 2 == 0 && ky == n2 / 2), nz = (n3 % 2 == 0 && kz == n3 / 2);
    if ((nx || ny || (nz && n3 > 1)) && igamma == 0) {
        for (int c = 0; c < 81; c++) g[c] = -s0[c];
        return 0;
    }
    if (((nx && ny) || (nx && nz) || (ny && nz)) && igamma >= 2) {
        for (int c = 0; c < 81; c++) g[c] = 0.0;
        return 0;
    }
    int bad = 0;
    double xk[3], D[9];
    spatial_freq(kx, ky, kz, n1, n2, n3, xk);
    if (igamma == 0) {
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) D[3 * i + j] = xk[i] * xk[j];
    } else if (igamma == 1) {
        const double twopi = 2.0 * EVP_PI;
        const double xi = twopi * (double)kx / (double)n1, xj = twopi * (double)ky / (double)n2,
                     xz = twopi * (double)kz / (double)n3;
        D[0] = 2.0 * (cos(xi) - 1.0);
        D[4] = 2.0 * (cos(xj) - 1.0);
        D[8] = 2.0 * (cos(xz) - 1.0);
        D[3] = -sin(xi) * sin(xj);
        D[6] = -sin(xi) * sin(xz);
        D[7] = -sin(xj) * sin(xz);
        D[1] = D[3];
        D[2] = D[6];
        D[5] = D[7];
    } else {
        // kmod = i/4 (1 + e^{i xk1})(1 + e^{i xk2})(1 + e^{i xk3}) tan(xk/2); D = Re(kmod kmod^*)
        double br = 0.0, bi = 0.25;
        for (int l = 0; l < 3; l++) {
            const double fr = 1.0 + cos(xk[l]), fi = sin(xk[l]);
            const double r = br * fr - bi * fi, im = br * fi + bi * fr;
            br = r;
            bi = im;
        }
        double kr[3], ki[3];
        for (int l = 0; l < 3; l++) {
            const double t = tan(xk[l] / 2.0);
            kr[l] = t * br;
            ki[l] = t * bi;
        }
        double im2 = 0.0;
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) {
                D[3 * i + j] = kr[i] * kr[j] + ki[i] * ki[j];
                const double dim = ki[i] * kr[j] - kr[i] * ki[j];
                im2 += dim * dim;
            }
        if (sqrt(im2) > 1.0e-7) bad = 1;
    }
    double a[9];
    if (kx == 0 && ky == 0 && kz == 0) {
        for (int c = 0; c < 9; c++) a[c] = 0.0;
    } else {
        double A[9];
        for (int i = 0; i < 3; i++)
            for (int k = 0; k < 3; k++) {
                double x = 0.0;
                for (int j = 0; j < 3; j++)
                    for (int l = 0; l < 3; l++) x += c0[((i * 3 + j) * 3 + k) * 3 + l] * D[3 * j + l];
                A[3 * i + k] = x;
            }
        if (inv3u(A, a) != 0) bad = 1;
    }
    for (int p = 0; p < 3; p++)
        for (int q = 0; q < 3; q++)
            for (int i = 0; i < 3; i++)
                for (int j = 0; j < 3; j++) g[((p * 3 + q) * 3 + i) * 3 + j] = -a[3 * p + i] * D[3 * q + j];
    if (igamma == 1) {
        // g <- -g1 : (c0 : g) four times, as two 9x9 products (the four-fold sum regrouped)
        double g1[81], t[81];
        for (int c = 0; c < 81; c++) g1[c] = g[c];
        for (int itt = 0; itt < 4; itt++) {
            for (int mn = 0; mn < 9; mn++)
                for (int kl = 0; kl < 9; kl++) {
                    double x = 0.0;
                    for (int op = 0; op < 9; op++) x += c0[mn * 9 + op] * g[op * 9 + kl];
                    t[mn * 9 + kl] = x;
                }
            for (int ij = 0; ij < 9; ij++)
                for (int kl = 0; kl < 9; kl++) {
                    double x = 0.0;
                    for (int mn = 0; mn < 9; mn++) x += g1[ij * 9 + mn] * t[mn * 9 + kl];
                    g[ij * 9 + kl] = -x;
                }
        }
    }
    return bad;
}

// Real-space origin value of the Green operator (mean over the full spectrum), used by the
// modified augmented Lagrangian (various_functions.f90:798-807).
__global__ void __launch_bounds__(kBlock) k_goperr0(Dev d, const double* __restrict__ c0g, const double* __restrict__ s0g,
                                                    int igamma) {
    __shared__ double c0[81], s0[81];
    for (int i = threadIdx.x; i < 81; i += blockDim.x) { c0[i] = c0g[i]; s0[i] = s0g[i]; }
    __syncthreads();
    const long long N = d.N;
    const int n1 = d.n1, n2 = d.n2, n3 = d.n3;
    double s[81];
#pragma unroll
    for (int c = 0; c < 81; c++) s[c] = 0.0;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < N; v += (long long)gridDim.x * blockDim.x) {
        const int kx = (int)(v % n1), ky = (int)((v / n1) % n2), kz = (int)(v / ((long long)n1 * n2));
        if (igamma != 0) {
            double g[81];
            if (goper_at(igamma, kx, ky, kz, n1, n2, n3, c0, s0, g) != 0) set_err(d.err, 4);
            for (int c = 0; c < 81; c++) s[c] += g[c];
            continue;
        }
        const bool nyq = (n1 % 2 == 0 && kx == n1 / 2) || (n2 % 2 == 0 && ky == n2 / 2) || (n3 % 2 == 0 && kz == n3 / 2 && n3 > 1);
        if (nyq) {
            for (int c = 0; c < 81; c++) s[c] += -s0[c];
            continue;
        }
        if (v == 0) continue;
        double xi[3], A[9], a[9];
        spatial_freq(kx, ky, kz, n1, n2, n3, xi);
        for (int i = 0; i < 3; i++)
            for (int k = 0; k < 3; k++) {
                double x = 0.0;
                for (int j = 0; j < 3; j++)
                    for (int l = 0; l < 3; l++) x += c0[((i * 3 + j) * 3 + k) * 3 + l] * (xi[j] * xi[l]);
                A[3 * i + k] = x;
            }
        if (inv3u(A, a) != 0) set_err(d.err, 1);
        for (int p = 0; p < 3; p++)
            for (int q = 0; q < 3; q++)
                for (int i = 0; i < 3; i++)
                    for (int j = 0; j < 3; j++) s[((p * 3 + q) * 3 + i) * 3 + j] += -a[3 * p + i] * (xi[q] * xi[j]);
    }
    reduce_store<81, 0>(s, nullptr, d.partials, d.red + OFF_G0, d.counters + CNT_G0, hw_vb());
}
void launch_goperr0(const Dev& d, const double* c0, const double* s0, int igamma, cudaStream_t st) {
    k_goperr0<<<d.grid, kBlock, 0, st>>>(d, c0, s0, igamma);
}

// form_G for IGAMMA 1 and 2 on the half spectrum, once per increment (c0 changes per increment)
__global__ void __launch_bounds__(kBlock) k_goper_tab(Dev d, const double* __restrict__ c0g, const double* __restrict__ s0g,
                                                      int igamma) {
    __shared__ double c0[81], s0[81];
    for (int i = threadIdx.x; i < 81; i += blockDim.x) { c0[i] = c0g[i]; s0[i] = s0g[i]; }
    __syncthreads();
    const int n1h = d.n1h, n2 = d.n2, n3 = d.n3;
    const long long P = (long long)n1h * n2 * n3;
    for (long long pt = blockIdx.x * (long long)blockDim.x + threadIdx.x; pt < P; pt += (long long)gridDim.x * blockDim.x) {
        const int kx = (int)(pt % n1h), j = (int)((pt / n1h) % n2), k3 = (int)(pt / ((long long)n1h * n2));
        double g[81];
        if (goper_at(igamma, kx, j, k3, d.n1, n2, n3, c0, s0, g) != 0) set_err(d.err, 4);
        for (int c = 0; c < 81; c++) d.goper[c * P + pt] = g[c];
    }
}
void launch_goper_tab(const Dev& d, const double* c0, const double* s0, int igamma, cudaStream_t st) {
    k_goper_tab<<<d.grid, kBlock, 0, st>>>(d, c0, s0, igamma);
}

}  // namespace evp
