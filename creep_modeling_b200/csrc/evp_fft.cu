// evp_fft.cu -- FP64 3-D FFT engine of the spectral equilibrium step.
//
// Replaces the FFTW C2C plans of fourier_functions.f90:69-336 (forward of the
// 9 PK1 fields, Green-operator product, inverse, real part / N) with a
// half-spectrum transform in five passes over HBM:
//   x: R2C by packing two voxel rows into one complex pencil (prologue computes
//      P' = J (sigma - <sigma>) F^{-T}, LS-EVPFFT.f90:256-269, in registers)
//   y: C2C
//   z: C2C forward -> Gamma(xi):P'(xi) evaluated on the fly from c0
//      (form_G igamma=0 + convolution_with_Goper, various_functions.f90:640-809,
//      999-1037) -> C2C inverse, one kernel, one read + one write of the spectrum
//   y: C2C inverse
//   x: C2R + epilogue (dvelgradref, and the F^{-1}-weighted average that
//      correction_to_current needs, various_functions.f90:1085-1101)
// Each pass stages pencils in shared memory and runs a mixed-radix Stockham
// FFT (radices 2,3,4,5,7,8,11,13) with twiddles from a per-axis table.
// The grid-update path (integrate_tensor2, various_functions.f90:359-429) reuses
// the same passes with a different z operator.
#include "evp_dev.cuh"
#include "evp_math.cuh"

#include <algorithm>
#include <cstdlib>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace evp {

// Complex arithmetic on double2 (FP64 path) and float2 (FP32 spectrum of the mixed-precision path).
template <class CT>
struct CxT;
template <>
struct CxT<double2> {
    using T = double;
};
template <>
struct CxT<float2> {
    using T = float;
};
template <class CT>
__device__ __forceinline__ CT mk(typename CxT<CT>::T x, typename CxT<CT>::T y) {
    CT r;
    r.x = x;
    r.y = y;
    return r;
}
template <class CT>
__device__ __forceinline__ CT cadd(CT a, CT b) { return mk<CT>(a.x + b.x, a.y + b.y); }
template <class CT>
__device__ __forceinline__ CT csub(CT a, CT b) { return mk<CT>(a.x - b.x, a.y - b.y); }
template <class CT>
__device__ __forceinline__ CT cmul(CT a, CT b) { return mk<CT>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
template <class CT>
__device__ __forceinline__ CT cconj(CT a) { return mk<CT>(a.x, -a.y); }
// multiply by -i (forward) or +i (inverse)
template <bool INV, class CT>
__device__ __forceinline__ CT mul_mi(CT a) { return INV ? mk<CT>(-a.y, a.x) : mk<CT>(a.y, -a.x); }

template <int R, bool INV, class CT>
__device__ __forceinline__ void dft_small(CT (&v)[R], const CT* __restrict__ tw, int n) {
    using T = typename CxT<CT>::T;
    if constexpr (R == 2) {
        CT a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if constexpr (R == 4) {
        CT t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]), t2 = cadd(v[1], v[3]), t3 = mul_mi<INV, CT>(csub(v[1], v[3]));
        v[0] = cadd(t0, t2);
        v[2] = csub(t0, t2);
        v[1] = cadd(t1, t3);
        v[3] = csub(t1, t3);
    } else if constexpr (R == 8) {
        const T c = (T)0.70710678118654752440;
        CT e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
        dft_small<4, INV, CT>(e, tw, n);
        dft_small<4, INV, CT>(o, tw, n);
        CT w1 = INV ? mk<CT>(c, c) : mk<CT>(c, -c);
        CT w3 = INV ? mk<CT>(-c, c) : mk<CT>(-c, -c);
        CT p0 = o[0], p1 = cmul(o[1], w1), p2 = mul_mi<INV, CT>(o[2]), p3 = cmul(o[3], w3);
        v[0] = cadd(e[0], p0); v[4] = csub(e[0], p0);
        v[1] = cadd(e[1], p1); v[5] = csub(e[1], p1);
        v[2] = cadd(e[2], p2); v[6] = csub(e[2], p2);
        v[3] = cadd(e[3], p3); v[7] = csub(e[3], p3);
    } else {
        CT in[R];
#pragma unroll
        for (int r = 0; r < R; r++) in[r] = v[r];
        const int step = n / R;
#pragma unroll
        for (int q = 0; q < R; q++) {
            CT acc = in[0];
#pragma unroll
            for (int r = 1; r < R; r++) {
                CT w = tw[((r * q) % R) * step];
                if (INV) w.y = -w.y;
                acc = cadd(acc, cmul(in[r], w));
            }
            v[q] = acc;
        }
    }
}

// One Stockham stage over P pencils of length n stored element-major in
// shared memory: element e of pencil p at s[e*ES + p].
template <int R, bool INV, int MAXB, class CT>
__device__ __forceinline__ void fft_stage(CT* s, int ES, int P, int n, int Ns, const CT* __restrict__ tw) {
    const int nb = n / R, total = nb * P;
    CT v[MAXB][R];
#pragma unroll
    for (int q = 0; q < MAXB; q++) {
        const int b = threadIdx.x + q * blockDim.x;
        if (b < total) {
            const int p = b % P, j = b / P;
#pragma unroll
            for (int r = 0; r < R; r++) v[q][r] = s[(j + r * nb) * ES + p];
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < MAXB; q++) {
        const int b = threadIdx.x + q * blockDim.x;
        if (b < total) {
            const int p = b % P, j = b / P, jm = j % Ns;
            const int step = jm * (n / (Ns * R));
#pragma unroll
            for (int r = 1; r < R; r++) {
                CT w = tw[r * step];
                if (INV) w.y = -w.y;
                v[q][r] = cmul(v[q][r], w);
            }
            dft_small<R, INV, CT>(v[q], tw, n);
            const int idxD = (j / Ns) * Ns * R + jm;
#pragma unroll
            for (int r = 0; r < R; r++) s[(idxD + r * Ns) * ES + p] = v[q][r];
        }
    }
    __syncthreads();
}

// Radix sets: RS = 0 compiles the power-of-two radices only (2, 4, 8), RS = 1
// every radix.  Butterflies per thread fall with the radix so that no stage
// holds more than 16 complex values per thread: two for every power-of-two
// radix with RS = 0; four for radices 2-4, two for 5-8 and one for 11 and 13
// with RS = 1.  Every kernel then fits 128 registers, two blocks of 256
// threads per SM; the launchers size blocks for the stage that needs the most
// threads (stage_threads).
__host__ __device__ constexpr int fft_maxb_r(int rs, int R) { return rs == 0 ? 2 : (R <= 4 ? 4 : (R <= 8 ? 2 : 1)); }

// An odd-radix stage as a function of its own (ODD_CALL in fft_run): its registers are
// then allocated apart from a kernel with a heavy epilogue (the grid-update z pass).
template <int R, bool INV, int MAXB, class CT>
__device__ __noinline__ void fft_stage_call(CT* s, int ES, int P, int n, int Ns, const CT* __restrict__ tw) {
    fft_stage<R, INV, MAXB, CT>(s, ES, P, n, Ns, tw);
}
template <int R, bool INV, int MAXB, class CT, bool CALL>
__device__ __forceinline__ void fft_stage_odd(CT* s, int ES, int P, int n, int Ns, const CT* __restrict__ tw) {
    if constexpr (CALL) fft_stage_call<R, INV, MAXB, CT>(s, ES, P, n, Ns, tw);
    else fft_stage<R, INV, MAXB, CT>(s, ES, P, n, Ns, tw);
}

template <bool INV, int RS, class CT, bool ODD_CALL = false>
__device__ void fft_run(CT* s, int ES, int P, const FftPlan1D& pl, const CT* __restrict__ tw) {
    int Ns = 1;
    for (int st = 0; st < pl.nst; st++) {
        const int R = pl.rad[st];
        switch (R) {
            case 2: fft_stage<2, INV, fft_maxb_r(RS, 2), CT>(s, ES, P, pl.n, Ns, tw); break;
            case 4: fft_stage<4, INV, fft_maxb_r(RS, 4), CT>(s, ES, P, pl.n, Ns, tw); break;
            case 8: fft_stage<8, INV, fft_maxb_r(RS, 8), CT>(s, ES, P, pl.n, Ns, tw); break;
            default:
                if constexpr (RS != 0) {
                    switch (R) {
                        case 3: fft_stage_odd<3, INV, fft_maxb_r(RS, 3), CT, ODD_CALL>(s, ES, P, pl.n, Ns, tw); break;
                        case 5: fft_stage_odd<5, INV, fft_maxb_r(RS, 5), CT, ODD_CALL>(s, ES, P, pl.n, Ns, tw); break;
                        case 7: fft_stage_odd<7, INV, fft_maxb_r(RS, 7), CT, ODD_CALL>(s, ES, P, pl.n, Ns, tw); break;
                        case 11: fft_stage_odd<11, INV, fft_maxb_r(RS, 11), CT, ODD_CALL>(s, ES, P, pl.n, Ns, tw); break;
                        case 13: fft_stage_odd<13, INV, fft_maxb_r(RS, 13), CT, ODD_CALL>(s, ES, P, pl.n, Ns, tw); break;
                        default: break;
                    }
                }
                break;
        }
        Ns *= R;
    }
}

FftPlan1D make_plan(int n) {
    FftPlan1D pl;
    pl.n = n;
    pl.nst = 0;
    int m = n, e2 = 0;
    while (m % 2 == 0) { m /= 2; e2++; }
    // powers of two: as many radix-8 as possible, a lone factor 2 turned into 4*4
    int n8 = e2 / 3, rem = e2 % 3, n4 = 0, n2 = 0;
    if (rem == 2) n4 = 1;
    else if (rem == 1) {
        if (n8 > 0) { n8--; n4 = 2; }
        else n2 = 1;
    }
    for (int i = 0; i < n8; i++) pl.rad[pl.nst++] = 8;
    for (int i = 0; i < n4; i++) pl.rad[pl.nst++] = 4;
    for (int i = 0; i < n2; i++) pl.rad[pl.nst++] = 2;
    const int odd[5] = {3, 5, 7, 11, 13};
    for (int f : odd)
        while (m % f == 0) {
            if (pl.nst >= 8) throw std::runtime_error("FFT length has too many factors: " + std::to_string(n));
            pl.rad[pl.nst++] = f;
            m /= f;
        }
    if (m != 1) throw std::runtime_error("unsupported FFT length " + std::to_string(n) + " (prime factors must be <= 13)");
    return pl;
}
// threads that cover every stage of the plan for `pencils` pencils (radix set rs)
static long long stage_threads(const FftPlan1D& pl, long long pencils, int rs) {
    long long t = 1;
    for (int i = 0; i < pl.nst; i++) {
        const int R = pl.rad[i], mb = fft_maxb_r(rs, R);
        const long long b = (pencils * (pl.n / R) + mb - 1) / mb;
        t = b > t ? b : t;
    }
    return t;
}

// twiddle table of an axis in the complex type of the pass
template <class CT>
__device__ __forceinline__ const CT* twid(const Dev& d, int axis);
template <>
__device__ __forceinline__ const double2* twid<double2>(const Dev& d, int axis) {
    return axis == 1 ? d.tw1 : (axis == 2 ? d.tw2 : d.tw3);
}
template <>
__device__ __forceinline__ const float2* twid<float2>(const Dev& d, int axis) {
    return axis == 1 ? d.tw1f : (axis == 2 ? d.tw2f : d.tw3f);
}

// ---------------------------------------------------------------- x forward (R2C)
// mode 0: P'_ij = J * ((sigma - <sigma>) F^{-T})_ij ; mode 1: (L F)_ij (grid update)
template <int RS, class CT>
__device__ __forceinline__ void body_fft_x_fwd(const Dev& d, const FftPlan1D& pl, int G, int mode, int sg_off, const VB& vb) {
    using Re = typename CxT<CT>::T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    CT* const s = reinterpret_cast<CT*>(smem_raw);
    CT* const spec = reinterpret_cast<CT*>(d.spec);
    const int n1 = d.n1, n1h = d.n1h;
    const long long N = d.N;
    const int nrows = d.n2 * d.n3;
    const int P = 9 * G;
    const int pair0 = vb.x * G;
    __shared__ double sga[6];
    if (mode == 0 && threadIdx.x < 6) sga[threadIdx.x] = __ldcg(&d.red[sg_off + threadIdx.x]);
    __syncthreads();
    for (int idx = threadIdx.x; idx < G * 2 * n1; idx += blockDim.x) {
        const int g = idx / (2 * n1), rem = idx % (2 * n1), half = rem / n1, x = rem % n1;
        const int row = 2 * (pair0 + g) + half;
        double val[9];
        if (row < nrows) {
            const long long v = (long long)row * n1 + x;
            if (mode == 0) {
                double sig[9], fi[9], a6[6];
#pragma unroll
                for (int c = 0; c < 6; c++) a6[c] = d.sg[c * N + v] - sga[c];
                s6_to_t2(a6, sig);
#pragma unroll
                for (int c = 0; c < 9; c++) fi[c] = d.Finv[c * N + v];
                const double J = d.detF[v];
                mm3_bt(sig, fi, val);
#pragma unroll
                for (int c = 0; c < 9; c++) val[c] = val[c] * J;
            } else {
                double L[9], F[9];
#pragma unroll
                for (int c = 0; c < 9; c++) { L[c] = d.velgrad[c * N + v]; F[c] = d.F[c * N + v]; }
                mm3(L, F, val);
            }
        } else {
#pragma unroll
            for (int c = 0; c < 9; c++) val[c] = 0.0;
        }
        Re* sd = reinterpret_cast<Re*>(s);
#pragma unroll
        for (int c = 0; c < 9; c++) sd[2 * (x * P + c * G + g) + half] = (Re)val[c];
    }
    __syncthreads();
    fft_run<false, RS, CT>(s, P, P, pl, twid<CT>(d, 1));
    // unpack the two real rows of every pencil
    for (int idx = threadIdx.x; idx < P * n1h; idx += blockDim.x) {
        const int k = idx % n1h, p = idx / n1h;
        const int c = p / G, g = p % G;
        const CT Z = s[k * P + p];
        const CT Zc = cconj(s[((n1 - k) % n1) * P + p]);
        const CT Xa = mk<CT>((Re)0.5 * (Z.x + Zc.x), (Re)0.5 * (Z.y + Zc.y));
        const CT dZ = csub(Z, Zc);
        const CT Xb = mk<CT>((Re)0.5 * dZ.y, (Re)-0.5 * dZ.x);
        const int ra = 2 * (pair0 + g);
        if (ra < nrows) spec[((long long)c * nrows + ra) * n1h + k] = Xa;
        if (ra + 1 < nrows) spec[((long long)c * nrows + ra + 1) * n1h + k] = Xb;
    }
}
template <int RS, class CT>
__global__ void __launch_bounds__(256, 2) k_fft_x_fwd(Dev d, FftPlan1D pl, int G, int mode, int sg_off) {
    body_fft_x_fwd<RS, CT>(d, pl, G, mode, sg_off, hw_vb());
}

// ---------------------------------------------------------------- y (C2C)
// TMA staging of pencils: nrows rows of ncol FP64 complex values (16 bytes each, so both
// ends of every row are 16-byte aligned), row r from global src(r) to shared dst(r), by bulk
// copies that complete on one mbarrier.  Thread 0 posts the expected byte count, then the 32
// lanes of warp 0 issue the rows; every thread waits for the bytes with a bounded wait (each
// try_wait suspends for a while before it fails; past the bound the error word gets bit 3 and
// the solve stops).  Callers zero the columns past the spectrum's edge with ordinary stores.
template <class SrcF, class DstF>
__device__ __forceinline__ void tma_rows(int nrows, int ncol, SrcF src, DstF dst, int* err) {
    __shared__ __align__(8) unsigned long long bar;
    const unsigned sbar = (unsigned)__cvta_generic_to_shared(&bar);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sbar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        if (threadIdx.x == 0) {
            const unsigned bytes = (unsigned)(nrows * ncol * 16);
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sbar), "r"(bytes) : "memory");
        }
        __syncwarp();
        for (int r = threadIdx.x; r < nrows; r += 32) {
            const unsigned d = (unsigned)__cvta_generic_to_shared(dst(r));
            asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(d),
                         "l"(src(r)), "r"((unsigned)(ncol * 16)), "r"(sbar)
                         : "memory");
        }
    }
    unsigned done = 0;
    for (long tries = 0; !done; tries++) {
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n\tselp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(done)
                     : "r"(sbar)
                     : "memory");
        if (!done && tries > (1L << 20)) {
            atomicOr(err, 8);
            break;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(sbar) : "memory");
}

template <bool INV, int RS, class CT>
__device__ __forceinline__ void body_fft_y(const Dev& d, const FftPlan1D& pl, int T, const VB& vb) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    CT* const s = reinterpret_cast<CT*>(smem_raw);
    const int n1h = d.n1h, n2 = d.n2, n3 = d.n3;
    const int kx0 = vb.x * T, k3 = vb.y, c = vb.z;
    CT* base = reinterpret_cast<CT*>(d.spec) + ((long long)c * n3 + k3) * n2 * n1h;
    if constexpr (sizeof(CT) == 16) {
        // FP64 spectrum: the block's pencils arrive by TMA bulk copies, one per y row (its valid columns)
        const int ncol = min(T, n1h - kx0);
        for (int idx = threadIdx.x; idx < (T - ncol) * n2; idx += blockDim.x) {
            const int t = ncol + idx % (T - ncol), j = idx / (T - ncol);
            s[j * T + t] = mk<CT>(0, 0);
        }
        tma_rows(n2, ncol, [&](int j) { return base + (long long)j * n1h + kx0; }, [&](int j) { return s + (size_t)j * T; },
                 d.err);
    } else {
        for (int idx = threadIdx.x; idx < T * n2; idx += blockDim.x) {
            const int t = idx % T, j = idx / T, kx = kx0 + t;
            s[j * T + t] = (kx < n1h) ? base[(long long)j * n1h + kx] : mk<CT>(0, 0);
        }
        __syncthreads();
    }
    fft_run<INV, RS, CT>(s, T, T, pl, twid<CT>(d, 2));
    for (int idx = threadIdx.x; idx < T * n2; idx += blockDim.x) {
        const int t = idx % T, j = idx / T, kx = kx0 + t;
        if (kx < n1h) base[(long long)j * n1h + kx] = s[j * T + t];
    }
}
template <bool INV, int RS, class CT>
__global__ void __launch_bounds__(256, 2) k_fft_y(Dev d, FftPlan1D pl, int T) { body_fft_y<INV, RS, CT>(d, pl, T, hw_vb()); }

// ---------------------------------------------------------------- z fused with the Green operator
__device__ __forceinline__ double xi_of(int k, int n) {
    const double twopi = 2.0 * EVP_PI;
    return (k + 1 <= n / 2) ? twopi * (double)k / (double)n : twopi * (double)(k - n) / (double)n;
}

// 3x3 inverse for the Green step: the FP64 path uses the LU inverse of the other
// kernels; the FP32 path the adjugate over the determinant (singular: returns 1).
__device__ __forceinline__ int inv3_any(const double* a, double* ai) { return inv3u(a, ai); }
__device__ __forceinline__ int inv3_any(const float* a, float* ai) {
    const float c00 = a[4] * a[8] - a[5] * a[7], c01 = a[5] * a[6] - a[3] * a[8], c02 = a[3] * a[7] - a[4] * a[6];
    const float det = a[0] * c00 + a[1] * c01 + a[2] * c02;
    if (det == 0.0f) return 1;
    const float r = 1.0f / det;
    ai[0] = c00 * r;
    ai[1] = (a[2] * a[7] - a[1] * a[8]) * r;
    ai[2] = (a[1] * a[5] - a[2] * a[4]) * r;
    ai[3] = c01 * r;
    ai[4] = (a[0] * a[8] - a[2] * a[6]) * r;
    ai[5] = (a[2] * a[3] - a[0] * a[5]) * r;
    ai[6] = c02 * r;
    ai[7] = (a[1] * a[6] - a[0] * a[7]) * r;
    ai[8] = (a[0] * a[4] - a[1] * a[3]) * r;
    return 0;
}

template <int RS, class CT>
__device__ __forceinline__ void body_fft_z_green(const Dev& d, const FftPlan1D& pl, int T, const double* __restrict__ c0g,
                                                 const double* __restrict__ s0g, const VB& vb) {
    using Re = typename CxT<CT>::T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    CT* const s = reinterpret_cast<CT*>(smem_raw);
    CT* const spec = reinterpret_cast<CT*>(d.spec);
    __shared__ Re c0[81], s0[81];
    const int n1 = d.n1, n2 = d.n2, n3 = d.n3, n1h = d.n1h;
    const int kx0 = vb.x * T, j = vb.y;
    const int P = 9 * T;
    for (int i = threadIdx.x; i < 81; i += blockDim.x) { c0[i] = (Re)c0g[i]; s0[i] = (Re)s0g[i]; }
    const long long plane = (long long)n2 * n1h;
    // ordinary loads: the block's rows are short (T complex values per component and z), which
    // suits TMA bulk copies badly (measured: 43 -> 68 us per 64^3 launch with one copy per row)
    for (int idx = threadIdx.x; idx < P * n3; idx += blockDim.x) {
        const int t = idx % T, r = idx / T, c = r % 9, k3 = r / 9, kx = kx0 + t;
        s[k3 * P + c * T + t] = (kx < n1h) ? spec[((long long)c * n3 + k3) * plane + (long long)j * n1h + kx] : mk<CT>(0, 0);
    }
    __syncthreads();
    fft_run<false, RS, CT>(s, P, P, pl, twid<CT>(d, 3));
    const bool nyq_y = (n2 % 2 == 0 && j == n2 / 2);
    const Re xiy = (Re)xi_of(j, n2);
    for (int idx = threadIdx.x; idx < T * n3; idx += blockDim.x) {
        const int t = idx % T, k3 = idx / T, kx = kx0 + t;
        if (kx >= n1h) continue;
        CT* q = s + k3 * P + t;
        CT a[9], r[9];
#pragma unroll
        for (int c = 0; c < 9; c++) a[c] = q[c * T];
        const bool nyq = (n1 % 2 == 0 && kx == n1 / 2) || nyq_y || (n3 % 2 == 0 && k3 == n3 / 2 && n3 > 1);
        if (d.gtab) {  // IGAMMA 1 or 2: the tabulated operator, r_pq = Gamma_pqij a_ij
            const long long P = (long long)n1h * n2 * n3, pt = ((long long)k3 * n2 + j) * n1h + kx;
#pragma unroll
            for (int pq = 0; pq < 9; pq++) {
                CT acc = mk<CT>(0, 0);
#pragma unroll
                for (int ij = 0; ij < 9; ij++) {
                    const Re g = (Re)d.goper[(pq * 9 + ij) * P + pt];
                    acc.x += g * a[ij].x;
                    acc.y += g * a[ij].y;
                }
                r[pq] = acc;
            }
        } else if (kx == 0 && j == 0 && k3 == 0) {
#pragma unroll
            for (int c = 0; c < 9; c++) r[c] = mk<CT>(0, 0);
        } else if (nyq) {
            // Nyquist planes: Gamma = -s0 (various_functions.f90:646-651)
#pragma unroll
            for (int c = 0; c < 9; c++) {
                CT acc = mk<CT>(0, 0);
#pragma unroll
                for (int e = 0; e < 9; e++) {
                    const Re g = -s0[c * 9 + e];
                    acc.x += g * a[e].x;
                    acc.y += g * a[e].y;
                }
                r[c] = acc;
            }
        } else {
            const Re xi[3] = {(Re)xi_of(kx, n1), xiy, (n3 == 1) ? (Re)0 : (Re)xi_of(k3, n3)};
            Re A[9], ai[9];
#pragma unroll
            for (int i = 0; i < 3; i++)
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    Re x = 0;
#pragma unroll
                    for (int jj = 0; jj < 3; jj++)
#pragma unroll
                        for (int l = 0; l < 3; l++) x += c0[((i * 3 + jj) * 3 + k) * 3 + l] * (xi[jj] * xi[l]);
                    A[3 * i + k] = x;
                }
            if (inv3_any(A, ai) != 0) atomicOr(d.err, 1);
            // r_ij = -xi_j * sum_k ai_ik (P xi)_k
            CT pv[3], wv[3];
#pragma unroll
            for (int k = 0; k < 3; k++) {
                CT acc = mk<CT>(0, 0);
#pragma unroll
                for (int l = 0; l < 3; l++) { acc.x += a[3 * k + l].x * xi[l]; acc.y += a[3 * k + l].y * xi[l]; }
                pv[k] = acc;
            }
#pragma unroll
            for (int i = 0; i < 3; i++) {
                CT acc = mk<CT>(0, 0);
#pragma unroll
                for (int k = 0; k < 3; k++) { acc.x += ai[3 * i + k] * pv[k].x; acc.y += ai[3 * i + k] * pv[k].y; }
                wv[i] = acc;
            }
#pragma unroll
            for (int i = 0; i < 3; i++)
#pragma unroll
                for (int jj = 0; jj < 3; jj++) r[3 * i + jj] = mk<CT>(-xi[jj] * wv[i].x, -xi[jj] * wv[i].y);
        }
#pragma unroll
        for (int c = 0; c < 9; c++) q[c * T] = r[c];
    }
    __syncthreads();
    fft_run<true, RS, CT>(s, P, P, pl, twid<CT>(d, 3));
    for (int idx = threadIdx.x; idx < P * n3; idx += blockDim.x) {
        const int t = idx % T, r = idx / T, c = r % 9, k3 = r / 9, kx = kx0 + t;
        if (kx < n1h) spec[((long long)c * n3 + k3) * plane + (long long)j * n1h + kx] = s[k3 * P + c * T + t];
    }
}
template <int RS, class CT>
__global__ void __launch_bounds__(256, 2) k_fft_z_green(Dev d, FftPlan1D pl, int T, const double* __restrict__ c0g,
                                                        const double* __restrict__ s0g) {
    body_fft_z_green<RS, CT>(d, pl, T, c0g, s0g, hw_vb());
}

// ---------------------------------------------------------------- z fused with the spectral integration (grid update)
template <int RS>
__global__ void __launch_bounds__(256, 2) k_fft_z_integ(Dev d, FftPlan1D pl, int T, int ideriv) {
    extern __shared__ double2 s[];
    const int n1 = d.n1, n2 = d.n2, n3 = d.n3, n1h = d.n1h;
    const int kx0 = blockIdx.x * T, j = blockIdx.y;
    const int P = 9 * T;
    const long long plane = (long long)n2 * n1h;
    for (int idx = threadIdx.x; idx < P * n3; idx += blockDim.x) {
        const int t = idx % T, r = idx / T, c = r % 9, k3 = r / 9, kx = kx0 + t;
        s[k3 * P + c * T + t] = (kx < n1h) ? d.spec[((long long)c * n3 + k3) * plane + (long long)j * n1h + kx] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    fft_run<false, RS, double2, true>(s, P, P, pl, d.tw3);
    if (blockIdx.x == 0 && j == 0 && threadIdx.x < 9) {
        const double2 z = s[threadIdx.x * T];
        d.red[OFF_DC + 2 * threadIdx.x] = z.x;
        d.red[OFF_DC + 2 * threadIdx.x + 1] = z.y;
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < T * n3; idx += blockDim.x) {
        const int t = idx % T, k3 = idx / T, kx = kx0 + t;
        if (kx >= n1h) continue;
        double2* q = s + k3 * P + t;
        double2 g[9];
#pragma unroll
        for (int c = 0; c < 9; c++) g[c] = q[c * T];
        const double xi[3] = {xi_of(kx, n1), xi_of(j, n2), (n3 == 1) ? 0.0 : xi_of(k3, n3)};
        double2 km[3];
        if (ideriv == 2) {
            // kmod = i/4 (1+e^{i xi1})(1+e^{i xi2})(1+e^{i xi3}) * tan(xi/2)
            double2 b = make_double2(0.0, 0.25);
            for (int l = 0; l < 3; l++) {
                double sn, cs;
                sincos(xi[l], &sn, &cs);
                b = cmul(b, make_double2(1.0 + cs, sn));
            }
            for (int l = 0; l < 3; l++) { const double tn = tan(xi[l] / 2.0); km[l] = make_double2(tn * b.x, tn * b.y); }
        } else {
            for (int l = 0; l < 3; l++) km[l] = make_double2(0.0, (ideriv == 0) ? xi[l] : sin(xi[l]));
        }
        const double kk = km[0].x * km[0].x + km[0].y * km[0].y + km[1].x * km[1].x + km[1].y * km[1].y + km[2].x * km[2].x +
                          km[2].y * km[2].y;
        double2 u[3];
        for (int l = 0; l < 3; l++) {
            double2 acc = make_double2(0.0, 0.0);
            if (kk > 0.0)
                for (int m = 0; m < 3; m++) {
                    const double2 t2 = cmul(cconj(km[m]), g[3 * l + m]);
                    acc = cadd(acc, make_double2(t2.x / kk, t2.y / kk));
                }
            u[l] = acc;
        }
        if (ideriv == 2 && (n1 % 2 == 0 && kx == n1 / 2) && (n2 % 2 == 0 && j == n2 / 2) && (n3 % 2 == 0 && k3 == n3 / 2 && n3 > 1))
            for (int l = 0; l < 3; l++) u[l] = make_double2(0.0, 0.0);
        for (int l = 0; l < 3; l++) q[l * T] = u[l];
    }
    __syncthreads();
    fft_run<true, RS, double2, true>(s, P, 3 * T, pl, d.tw3);
    for (int idx = threadIdx.x; idx < 3 * T * n3; idx += blockDim.x) {
        const int t = idx % T, r = idx / T, c = r % 3, k3 = r / 3, kx = kx0 + t;
        if (kx < n1h) d.spec[((long long)c * n3 + k3) * plane + (long long)j * n1h + kx] = s[k3 * P + c * T + t];
    }
}

// ---------------------------------------------------------------- z fused with the spectral gradient (IDISPINI start-up)
// The spectrum holds 9 components with component 3m + l = u_l; each is multiplied by the
// derivative symbol of direction m (ideriv 1: i sin(xi), 2: the rotated-scheme kmod, zero at the
// point where all three Nyquist planes meet), so the inverse gives d u_l / d x_m
// (gradient_tensor1, various_functions.f90:56-112).
template <int RS>
__global__ void __launch_bounds__(256, 2) k_fft_z_grad(Dev d, FftPlan1D pl, int T, int ideriv) {
    extern __shared__ double2 s[];
    const int n1 = d.n1, n2 = d.n2, n3 = d.n3, n1h = d.n1h;
    const int kx0 = blockIdx.x * T, j = blockIdx.y;
    const int P = 9 * T;
    const long long plane = (long long)n2 * n1h;
    for (int idx = threadIdx.x; idx < P * n3; idx += blockDim.x) {
        const int t = idx % T, r = idx / T, c = r % 9, k3 = r / 9, kx = kx0 + t;
        s[k3 * P + c * T + t] = (kx < n1h) ? d.spec[((long long)c * n3 + k3) * plane + (long long)j * n1h + kx] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    fft_run<false, RS, double2>(s, P, P, pl, d.tw3);
    __syncthreads();
    for (int idx = threadIdx.x; idx < T * n3; idx += blockDim.x) {
        const int t = idx % T, k3 = idx / T, kx = kx0 + t;
        if (kx >= n1h) continue;
        double2* q = s + k3 * P + t;
        const double xi[3] = {xi_of(kx, n1), xi_of(j, n2), (n3 == 1) ? 0.0 : xi_of(k3, n3)};
        double2 km[3];
        if (ideriv == 2) {
            double2 b = make_double2(0.0, 0.25);
            for (int l = 0; l < 3; l++) {
                double sn, cs;
                sincos(xi[l], &sn, &cs);
                b = cmul(b, make_double2(1.0 + cs, sn));
            }
            for (int l = 0; l < 3; l++) { const double tn = tan(xi[l] / 2.0); km[l] = make_double2(tn * b.x, tn * b.y); }
        } else {
            for (int l = 0; l < 3; l++) km[l] = make_double2(0.0, (ideriv == 0) ? xi[l] : sin(xi[l]));
        }
        const bool zero = ideriv == 2 && (n1 % 2 == 0 && kx == n1 / 2) && (n2 % 2 == 0 && j == n2 / 2) &&
                          (n3 % 2 == 0 && k3 == n3 / 2 && n3 > 1);
#pragma unroll
        for (int m = 0; m < 3; m++)
#pragma unroll
            for (int l = 0; l < 3; l++) {
                const int c = 3 * m + l;
                q[c * T] = zero ? make_double2(0.0, 0.0) : cmul(q[c * T], km[m]);
            }
    }
    __syncthreads();
    fft_run<true, RS, double2>(s, P, P, pl, d.tw3);
    for (int idx = threadIdx.x; idx < P * n3; idx += blockDim.x) {
        const int t = idx % T, r = idx / T, c = r % 9, k3 = r / 9, kx = kx0 + t;
        if (kx < n1h) d.spec[((long long)c * n3 + k3) * plane + (long long)j * n1h + kx] = s[k3 * P + c * T + t];
    }
}

// ---------------------------------------------------------------- x inverse (C2R)
template <int RS, class CT>
__device__ __forceinline__ void body_fft_x_inv(const Dev& d, const FftPlan1D& pl, int G, int ncomp, int mode, const XinvParams& xp,
                                               const VB& vb) {
    using Re = typename CxT<CT>::T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    CT* const s = reinterpret_cast<CT*>(smem_raw);
    const CT* const spec = reinterpret_cast<const CT*>(d.spec);
    const int n1 = d.n1, n1h = d.n1h;
    const long long N = d.N;
    const int nrows = d.n2 * d.n3;
    const int P = ncomp * G;
    const int pair0 = vb.x * G;
    const bool even = (n1 % 2 == 0);
    for (int idx = threadIdx.x; idx < P * n1; idx += blockDim.x) {
        const int x = idx % n1, p = idx / n1;
        const int c = p / G, g = p % G;
        const int ra = 2 * (pair0 + g);
        const int k = (x <= n1 / 2) ? x : n1 - x;
        const bool cj = (x > n1 / 2);
        CT A = mk<CT>(0, 0), B = mk<CT>(0, 0);
        if (ra < nrows) A = spec[((long long)c * nrows + ra) * n1h + k];
        if (ra + 1 < nrows) B = spec[((long long)c * nrows + ra + 1) * n1h + k];
        if (k == 0 || (even && k == n1 / 2)) { A.y = 0; B.y = 0; }
        if (cj) { A.y = -A.y; B.y = -B.y; }
        s[x * P + p] = mk<CT>(A.x - B.y, A.y + B.x);
    }
    __syncthreads();
    fft_run<true, RS, CT>(s, P, P, pl, twid<CT>(d, 1));
    const double invN = 1.0 / (double)N;
    double acc[9];
#pragma unroll
    for (int c = 0; c < 9; c++) acc[c] = 0.0;
    for (int idx = threadIdx.x; idx < G * 2 * n1; idx += blockDim.x) {
        const int g = idx / (2 * n1), rem = idx % (2 * n1), half = rem / n1, x = rem % n1;
        const int row = 2 * (pair0 + g) + half;
        if (row >= nrows) continue;
        const long long v = (long long)row * n1 + x;
        const Re* sd = reinterpret_cast<const Re*>(s);
        if (mode == 0) {
            double t[9], fi[9], u[9];
#pragma unroll
            for (int c = 0; c < 9; c++) {
                t[c] = (double)sd[2 * (x * P + c * G + g) + half] / (double)N;
                d.dvr[c * N + v] = t[c];
                fi[c] = d.Finv[c * N + v];
            }
            mm3(t, fi, u);
            const double w = d.wgtc[v];
#pragma unroll
            for (int c = 0; c < 9; c++) acc[c] += w * u[c];
        } else {
            for (int c = 0; c < ncomp; c++) d.dv3[c * N + v] = (double)sd[2 * (x * P + c * G + g) + half] / (double)N;
        }
    }
    (void)invN;
    if (mode != 0) return;
    // block partials -> the last block forms du = (dvelgradavg - <dL_ref F^{-1}>) inv(<F^{-1}>)
    __shared__ double sh[9][32];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int f = 0; f < 9; f++) {
        double x = acc[f];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) sh[f][warp] = x;
    }
    __syncthreads();
    if (warp == 0) {
        for (int f = 0; f < 9; f++) {
            double x = lane < nw ? sh[f][lane] : 0.0;
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            if (lane == 0) d.partials[(size_t)f * vb.nx + vb.x] = x;
        }
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = (atomicAdd(d.counters + CNT_XINV, 1u) == (unsigned)vb.nx - 1u);
    __syncthreads();
    __shared__ double fsum[9];
    if (last) {  // fold the block partials: one warp per field, fixed order
        __threadfence();
        for (int f = warp; f < 9; f += nw) {
            const double x = fold_sum(d.partials, vb.nx, f, lane);
            if (lane == 0) fsum[f] = x;
        }
        __syncthreads();
    }
    if (last && threadIdx.x == 0) {
        double fl[9], dd[9], du[9];
        for (int f = 0; f < 9; f++) {
            fl[f] = fsum[f];
            dd[f] = xp.dvelgradavg[f] - fl[f];
        }
        mm3(dd, xp.dinv, du);
        for (int f = 0; f < 9; f++) d.red[OFF_DU + f] = du[f];
        d.counters[CNT_XINV] = 0;
    }
}
template <int RS, class CT>
__global__ void __launch_bounds__(256, 2) k_fft_x_inv(Dev d, FftPlan1D pl, int G, int ncomp, int mode, XinvParams xp) {
    body_fft_x_inv<RS, CT>(d, pl, G, ncomp, mode, xp, hw_vb());
}

// ---------------------------------------------------------------- standalone Green-operator application
// x passes of evp_green_apply: the 9 real input fields come straight from a
// caller-owned array tau[c*N + v] and the result goes to out[c*N + v].
template <int RS>
__global__ void __launch_bounds__(256, 2) k_green_x_fwd(Dev d, FftPlan1D pl, int G, const double* __restrict__ tau) {
    extern __shared__ double2 s[];
    const int n1 = d.n1, n1h = d.n1h;
    const long long N = d.N;
    const int nrows = d.n2 * d.n3;
    const int P = 9 * G;
    const int pair0 = blockIdx.x * G;
    double* sd = reinterpret_cast<double*>(s);
    for (int idx = threadIdx.x; idx < G * 2 * n1; idx += blockDim.x) {
        const int g = idx / (2 * n1), rem = idx % (2 * n1), half = rem / n1, x = rem % n1;
        const int row = 2 * (pair0 + g) + half;
        const long long v = (long long)row * n1 + x;
#pragma unroll
        for (int c = 0; c < 9; c++) sd[2 * (x * P + c * G + g) + half] = (row < nrows) ? tau[c * N + v] : 0.0;
    }
    __syncthreads();
    fft_run<false, RS, double2>(s, P, P, pl, d.tw1);
    for (int idx = threadIdx.x; idx < P * n1h; idx += blockDim.x) {
        const int k = idx % n1h, p = idx / n1h;
        const int c = p / G, g = p % G;
        const double2 Z = s[k * P + p];
        const double2 Zc = cconj(s[((n1 - k) % n1) * P + p]);
        const double2 dZ = csub(Z, Zc);
        const int ra = 2 * (pair0 + g);
        if (ra < nrows) d.spec[((long long)c * nrows + ra) * n1h + k] = make_double2(0.5 * (Z.x + Zc.x), 0.5 * (Z.y + Zc.y));
        if (ra + 1 < nrows) d.spec[((long long)c * nrows + ra + 1) * n1h + k] = make_double2(0.5 * dZ.y, -0.5 * dZ.x);
    }
}
template <int RS>
__global__ void __launch_bounds__(256, 2) k_green_x_inv(Dev d, FftPlan1D pl, int G, double* __restrict__ out) {
    extern __shared__ double2 s[];
    const int n1 = d.n1, n1h = d.n1h;
    const long long N = d.N;
    const int nrows = d.n2 * d.n3;
    const int P = 9 * G;
    const int pair0 = blockIdx.x * G;
    const bool even = (n1 % 2 == 0);
    for (int idx = threadIdx.x; idx < P * n1; idx += blockDim.x) {
        const int x = idx % n1, p = idx / n1;
        const int c = p / G, g = p % G;
        const int ra = 2 * (pair0 + g);
        const int k = (x <= n1 / 2) ? x : n1 - x;
        double2 A = make_double2(0.0, 0.0), B = make_double2(0.0, 0.0);
        if (ra < nrows) A = d.spec[((long long)c * nrows + ra) * n1h + k];
        if (ra + 1 < nrows) B = d.spec[((long long)c * nrows + ra + 1) * n1h + k];
        if (k == 0 || (even && k == n1 / 2)) { A.y = 0.0; B.y = 0.0; }
        if (x > n1 / 2) { A.y = -A.y; B.y = -B.y; }
        s[x * P + p] = make_double2(A.x - B.y, A.y + B.x);
    }
    __syncthreads();
    fft_run<true, RS, double2>(s, P, P, pl, d.tw1);
    const double* sd = reinterpret_cast<const double*>(s);
    for (int idx = threadIdx.x; idx < G * 2 * n1; idx += blockDim.x) {
        const int g = idx / (2 * n1), rem = idx % (2 * n1), half = rem / n1, x = rem % n1;
        const int row = 2 * (pair0 + g) + half;
        if (row >= nrows) continue;
        const long long v = (long long)row * n1 + x;
#pragma unroll
        for (int c = 0; c < 9; c++) out[c * N + v] = sd[2 * (x * P + c * G + g) + half] / (double)N;
    }
}

// ---------------------------------------------------------------- launchers
// A pass needs, for P pencils of length n, the largest over its stages of
// P * (n / R) / (butterflies per thread at radix R) threads.  Each launcher picks the power-of-two kernels when the
// plan has only radices 2, 4 and 8, asks the kernel for its block-size limit
// (set by its register use) and shrinks its tile (pencils per block) until
// the threads fit.
static bool plan_pow2(const FftPlan1D& pl) {
    for (int i = 0; i < pl.nst; i++)
        if (pl.rad[i] != 2 && pl.rad[i] != 4 && pl.rad[i] != 8) return false;
    return true;
}
static int kernel_max_threads(const void* k) {
    cudaFuncAttributes a{};
    if (cudaFuncGetAttributes(&a, k) != cudaSuccess || a.maxThreadsPerBlock < 32) return 256;
    return a.maxThreadsPerBlock;
}
// largest tile T <= T0 whose ncomp * T pencils fit in maxthr threads; thr gets the block size
static int fit_tile(int T0, int ncomp, const FftPlan1D& pl, int rs, int want, int maxthr, int& thr) {
    for (int T = T0; T >= 1; T--) {
        const long long need = stage_threads(pl, (long long)ncomp * T, rs);
        int t = want > need ? want : (int)need;
        t = (t + 31) / 32 * 32;
        if (t > maxthr) t = maxthr / 32 * 32;
        if (need <= t) {
            thr = t;
            return T;
        }
    }
    throw std::runtime_error("FFT pencils of length " + std::to_string(pl.n) + " do not fit one block");
}
static int x_rows_per_block(int n1) { return (256 / n1) > 1 ? 256 / n1 : 1; }

static int sm_count() {
    static const int n = [] {
        int dev = 0, c = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, dev);
        return c < 1 ? 1 : c;
    }();
    return n;
}
// Tile choice: among tiles T <= T0 that fit (fit_tile), take the one with the
// least (waves of blocks) x (T + 1): block time grows with T, and a last wave
// that is mostly empty costs as much as a full one.
template <class BlocksOf, class SmemOf>
static int choose_tile(const void* kern, int T0, int ncomp, const FftPlan1D& pl, int rs, int want, int maxthr, BlocksOf blocks_of,
                       SmemOf smem_of, int& thr) {
    int best = -1, best_thr = 0;
    double best_cost = 0.0;
    for (int T = T0; T >= 1; T--) {
        int t = 0;
        if (fit_tile(T, ncomp, pl, rs, want, maxthr, t) != T) continue;
        int per_sm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, t, smem_of(T)) != cudaSuccess || per_sm < 1) continue;
        const long long slots = (long long)per_sm * sm_count();
        const long long waves = (blocks_of(T) + slots - 1) / slots;
        const double cost = (double)waves * (T + 1);
        if (best < 0 || cost < best_cost) {
            best = T;
            best_cost = cost;
            best_thr = t;
        }
    }
    if (best < 0) return fit_tile(T0, ncomp, pl, rs, want, maxthr, thr);
    thr = best_thr;
    return best;
}

template <int RS>
static void green_apply_rs(const Dev& d, const FftPlan1D& pl1, const FftPlan1D& pl2, const FftPlan1D& pl3, const double* tau,
                           double* out, const double* c0, const double* s0, cudaStream_t st) {
    static const int mx = std::min(kernel_max_threads((const void*)k_green_x_fwd<RS>), kernel_max_threads((const void*)k_green_x_inv<RS>));
    int thr = 0;
    const int G = fit_tile(x_rows_per_block(d.n1), 9, pl1, RS, 256, mx, thr);
    const int nrows = d.n2 * d.n3, npairs = (nrows + 1) / 2;
    const int grid = (npairs + G - 1) / G;
    const size_t smem = (size_t)9 * G * d.n1 * sizeof(double2);
    k_green_x_fwd<RS><<<grid, thr, smem, st>>>(d, pl1, G, tau);
    launch_fft_y(d, pl2, 9, false, st, 0);
    launch_fft_z_green(d, pl3, c0, s0, st, 0);
    launch_fft_y(d, pl2, 9, true, st, 0);
    k_green_x_inv<RS><<<grid, thr, smem, st>>>(d, pl1, G, out);
}
void launch_green_apply(const Dev& d, const FftPlan1D& pl1, const FftPlan1D& pl2, const FftPlan1D& pl3, const double* tau,
                        double* out, const double* c0, const double* s0, cudaStream_t st) {
    if (plan_pow2(pl1)) green_apply_rs<0>(d, pl1, pl2, pl3, tau, out, c0, s0, st);
    else green_apply_rs<1>(d, pl1, pl2, pl3, tau, out, c0, s0, st);
}

// ---------------------------------------------------------------- measured tile choice (autotuner)
// For the spectral passes whose work per pencil does not depend on the tile (x forward,
// y, z with the Green operator: no reduction inside), the tile is picked by timing the
// candidates on the device.  fft_autotune does that for a solve's grid at open time, once
// per grid and process (a few milliseconds); with a tile cache file (the executable's
// --fftw_save path, the server's tune_cache) the choices are also appended to the file and
// read back by later processes instead of timing again.  The occupancy / wave-count model
// gives the candidates' upper bound and the tile of the passes that are not tuned.  The
// tile does not change any result: every pencil is transformed by the same arithmetic.
struct TuneKey {
    int pass, rs, ct, n1, n2, n3;
    bool operator<(const TuneKey& o) const {
        const int a[6] = {pass, rs, ct, n1, n2, n3}, b[6] = {o.pass, o.rs, o.ct, o.n1, o.n2, o.n3};
        for (int i = 0; i < 6; i++)
            if (a[i] != b[i]) return a[i] < b[i];
        return false;
    }
};
enum : int { TUNE_XFWD = 0, TUNE_Y = 1, TUNE_ZGREEN = 2 };
static std::mutex g_tune_m;
static std::map<TuneKey, int> g_tuned;
static std::string g_tune_path;

static int tuned_tile(int pass, int rs, int ct, const Dev& d) {
    std::lock_guard<std::mutex> lk(g_tune_m);
    auto it = g_tuned.find(TuneKey{pass, rs, ct, d.n1, d.n2, d.n3});
    return it == g_tuned.end() ? -1 : it->second;
}

void fft_tune_cache(const std::string& path) {
    std::lock_guard<std::mutex> lk(g_tune_m);
    g_tune_path = path;
    if (path.empty()) return;
    std::ifstream f(path);
    std::string line;
    while (std::getline(f, line)) {  // "evp-tile pass rs ct n1 n2 n3 tile"
        std::istringstream is(line);
        std::string tag;
        TuneKey k{};
        int t = 0;
        if ((is >> tag >> k.pass >> k.rs >> k.ct >> k.n1 >> k.n2 >> k.n3 >> t) && tag == "evp-tile" && t > 0) g_tuned[k] = t;
    }
}

// Launch shape of one pass over one solve: grid (gx, gy, gz), tile (rows or pencils per
// block), threads per block and dynamic shared memory.  The single-solve launchers and the
// batched launches use the same shapes, so a solve's blocks do the same work either way.
struct FftShape {
    int gx, gy, gz, tile, thr;
    size_t smem;
};
template <int RS, class CT>
static FftShape x_fwd_shape(const Dev& d, const FftPlan1D& pl) {
    static const int mx = kernel_max_threads((const void*)k_fft_x_fwd<RS, CT>);
    int thr = 0;
    const long long npr = ((long long)d.n2 * d.n3 + 1) / 2;
    const int tt = tuned_tile(TUNE_XFWD, RS, sizeof(CT) == sizeof(float2), d);
    const int G = tt > 0 ? fit_tile(tt, 9, pl, RS, 128, mx, thr)
                         : choose_tile((const void*)k_fft_x_fwd<RS, CT>, x_rows_per_block(d.n1), 9, pl, RS, 128, mx,
                                       [&](int g) { return (npr + g - 1) / g; },
                                       [&](int g) { return (size_t)9 * g * d.n1 * sizeof(CT); }, thr);
    const int nrows = d.n2 * d.n3, npairs = (nrows + 1) / 2;
    return FftShape{(npairs + G - 1) / G, 1, 1, G, thr, (size_t)9 * G * d.n1 * sizeof(CT)};
}
template <int RS, class CT>
static void x_fwd_rs(const Dev& d, const FftPlan1D& pl, int mode, int sg_off, cudaStream_t st) {
    const FftShape sh = x_fwd_shape<RS, CT>(d, pl);
    k_fft_x_fwd<RS, CT><<<sh.gx, sh.thr, sh.smem, st>>>(d, pl, sh.tile, mode, sg_off);
}
void launch_fft_x_fwd(const Dev& d, const FftPlan1D& pl, int mode, int sg_off, cudaStream_t st, int prec) {
    const bool f32 = prec != 0 && mode == 0;  // the grid-update chain (mode 1) stays FP64
    if (plan_pow2(pl)) f32 ? x_fwd_rs<0, float2>(d, pl, mode, sg_off, st) : x_fwd_rs<0, double2>(d, pl, mode, sg_off, st);
    else f32 ? x_fwd_rs<1, float2>(d, pl, mode, sg_off, st) : x_fwd_rs<1, double2>(d, pl, mode, sg_off, st);
}

static int y_tile(const Dev& d) {
    const int budget = 40 * 1024;
    int nt = (int)(((long long)d.n1h * d.n2 * 16 + budget - 1) / budget);
    if (nt < 1) nt = 1;
    return (d.n1h + nt - 1) / nt;
}
template <int RS, class CT>
static FftShape y_shape(const Dev& d, const FftPlan1D& pl, int ncomp) {
    static const int mx = std::min(kernel_max_threads((const void*)k_fft_y<true, RS, CT>), kernel_max_threads((const void*)k_fft_y<false, RS, CT>));
    int thr = 0;
    const int tt = ncomp == 9 ? tuned_tile(TUNE_Y, RS, sizeof(CT) == sizeof(float2), d) : -1;
    const int T = tt > 0 ? fit_tile(tt, 1, pl, RS, 64, mx, thr)
                         : choose_tile((const void*)k_fft_y<false, RS, CT>, y_tile(d), 1, pl, RS, 64, mx,
                                       [&](int t) { return (long long)((d.n1h + t - 1) / t) * d.n3 * ncomp; },
                                       [&](int t) { return (size_t)t * d.n2 * sizeof(CT); }, thr);
    return FftShape{(d.n1h + T - 1) / T, d.n3, ncomp, T, thr, (size_t)T * d.n2 * sizeof(CT)};
}
template <int RS, class CT>
static void y_rs(const Dev& d, const FftPlan1D& pl, int ncomp, bool inverse, cudaStream_t st) {
    const FftShape sh = y_shape<RS, CT>(d, pl, ncomp);
    dim3 grid(sh.gx, sh.gy, sh.gz);
    if (inverse) k_fft_y<true, RS, CT><<<grid, sh.thr, sh.smem, st>>>(d, pl, sh.tile);
    else k_fft_y<false, RS, CT><<<grid, sh.thr, sh.smem, st>>>(d, pl, sh.tile);
}
void launch_fft_y(const Dev& d, const FftPlan1D& pl, int ncomp, bool inverse, cudaStream_t st, int prec) {
    if (plan_pow2(pl)) prec ? y_rs<0, float2>(d, pl, ncomp, inverse, st) : y_rs<0, double2>(d, pl, ncomp, inverse, st);
    else prec ? y_rs<1, float2>(d, pl, ncomp, inverse, st) : y_rs<1, double2>(d, pl, ncomp, inverse, st);
}

static int z_tile(const Dev& d) {
    const int budget = 72 * 1024;
    int nt = (int)(((long long)d.n1h * 9 * d.n3 * 16 + budget - 1) / budget);
    if (nt < 1) nt = 1;
    return (d.n1h + nt - 1) / nt;
}
template <int RS, class CT>
static FftShape z_green_shape(const Dev& d, const FftPlan1D& pl) {
    static const int mx = kernel_max_threads((const void*)k_fft_z_green<RS, CT>);
    int thr = 0;
    const int tt = tuned_tile(TUNE_ZGREEN, RS, sizeof(CT) == sizeof(float2), d);
    const int T = tt > 0 ? fit_tile(tt, 9, pl, RS, 128, mx, thr)
                         : choose_tile((const void*)k_fft_z_green<RS, CT>, z_tile(d), 9, pl, RS, 128, mx,
                                       [&](int t) { return (long long)((d.n1h + t - 1) / t) * d.n2; },
                                       [&](int t) { return (size_t)9 * t * d.n3 * sizeof(CT); }, thr);
    return FftShape{(d.n1h + T - 1) / T, d.n2, 1, T, thr, (size_t)9 * T * d.n3 * sizeof(CT)};
}
template <int RS, class CT>
static void z_green_rs(const Dev& d, const FftPlan1D& pl, const double* c0, const double* s0, cudaStream_t st) {
    const FftShape sh = z_green_shape<RS, CT>(d, pl);
    k_fft_z_green<RS, CT><<<dim3(sh.gx, sh.gy), sh.thr, sh.smem, st>>>(d, pl, sh.tile, c0, s0);
}
void launch_fft_z_green(const Dev& d, const FftPlan1D& pl, const double* c0, const double* s0, cudaStream_t st, int prec) {
    if (plan_pow2(pl)) prec ? z_green_rs<0, float2>(d, pl, c0, s0, st) : z_green_rs<0, double2>(d, pl, c0, s0, st);
    else prec ? z_green_rs<1, float2>(d, pl, c0, s0, st) : z_green_rs<1, double2>(d, pl, c0, s0, st);
}
template <int RS>
static void z_integ_rs(const Dev& d, const FftPlan1D& pl, int ideriv, cudaStream_t st) {
    static const int mx = kernel_max_threads((const void*)k_fft_z_integ<RS>);
    int thr = 0;
    const int T = choose_tile((const void*)k_fft_z_integ<RS>, z_tile(d), 9, pl, RS, 128, mx,
                              [&](int t) { return (long long)((d.n1h + t - 1) / t) * d.n2; },
                              [&](int t) { return (size_t)9 * t * d.n3 * sizeof(double2); }, thr);
    dim3 grid((d.n1h + T - 1) / T, d.n2);
    const size_t smem = (size_t)9 * T * d.n3 * sizeof(double2);
    k_fft_z_integ<RS><<<grid, thr, smem, st>>>(d, pl, T, ideriv);
}
void launch_fft_z_integ(const Dev& d, const FftPlan1D& pl, int ideriv, cudaStream_t st) {
    if (plan_pow2(pl)) z_integ_rs<0>(d, pl, ideriv, st);
    else z_integ_rs<1>(d, pl, ideriv, st);
}

template <int RS>
static void z_grad_rs(const Dev& d, const FftPlan1D& pl, int ideriv, cudaStream_t st) {
    static const int mx = kernel_max_threads((const void*)k_fft_z_grad<RS>);
    int thr = 0;
    const int T = choose_tile((const void*)k_fft_z_grad<RS>, z_tile(d), 9, pl, RS, 128, mx,
                              [&](int t) { return (long long)((d.n1h + t - 1) / t) * d.n2; },
                              [&](int t) { return (size_t)9 * t * d.n3 * sizeof(double2); }, thr);
    dim3 grid((d.n1h + T - 1) / T, d.n2);
    const size_t smem = (size_t)9 * T * d.n3 * sizeof(double2);
    k_fft_z_grad<RS><<<grid, thr, smem, st>>>(d, pl, T, ideriv);
}
template <int RS>
static void gradient_rs(const Dev& d, const FftPlan1D& pl1, const FftPlan1D& pl2, const FftPlan1D& pl3, const double* u9,
                        double* out, int ideriv, cudaStream_t st) {
    static const int mx = std::min(kernel_max_threads((const void*)k_green_x_fwd<RS>), kernel_max_threads((const void*)k_green_x_inv<RS>));
    int thr = 0;
    const int G = fit_tile(x_rows_per_block(d.n1), 9, pl1, RS, 256, mx, thr);
    const int nrows = d.n2 * d.n3, npairs = (nrows + 1) / 2;
    const int grid = (npairs + G - 1) / G;
    const size_t smem = (size_t)9 * G * d.n1 * sizeof(double2);
    k_green_x_fwd<RS><<<grid, thr, smem, st>>>(d, pl1, G, u9);
    launch_fft_y(d, pl2, 9, false, st, 0);
    if (plan_pow2(pl3)) z_grad_rs<0>(d, pl3, ideriv, st);
    else z_grad_rs<1>(d, pl3, ideriv, st);
    launch_fft_y(d, pl2, 9, true, st, 0);
    k_green_x_inv<RS><<<grid, thr, smem, st>>>(d, pl1, G, out);
}
void launch_gradient(const Dev& d, const FftPlan1D& pl1, const FftPlan1D& pl2, const FftPlan1D& pl3, const double* u9,
                     double* out, int ideriv, cudaStream_t st) {
    if (plan_pow2(pl1)) gradient_rs<0>(d, pl1, pl2, pl3, u9, out, ideriv, st);
    else gradient_rs<1>(d, pl1, pl2, pl3, u9, out, ideriv, st);
}
template <int RS, class CT>
static FftShape x_inv_shape(const Dev& d, const FftPlan1D& pl, int ncomp) {
    static const int mx = kernel_max_threads((const void*)k_fft_x_inv<RS, CT>);
    int thr = 0;
    const long long npr = ((long long)d.n2 * d.n3 + 1) / 2;
    const int G = choose_tile((const void*)k_fft_x_inv<RS, CT>, x_rows_per_block(d.n1), ncomp, pl, RS, 128, mx,
                              [&](int g) { return (npr + g - 1) / g; },
                              [&](int g) { return (size_t)ncomp * g * d.n1 * sizeof(CT); }, thr);
    const int nrows = d.n2 * d.n3, npairs = (nrows + 1) / 2;
    return FftShape{(npairs + G - 1) / G, 1, 1, G, thr, (size_t)ncomp * G * d.n1 * sizeof(CT)};
}
template <int RS, class CT>
static void x_inv_rs(const Dev& d, const FftPlan1D& pl, int mode, const XinvParams& p, cudaStream_t st) {
    const int ncomp = (mode == 0) ? 9 : 3;
    const FftShape sh = x_inv_shape<RS, CT>(d, pl, ncomp);
    k_fft_x_inv<RS, CT><<<sh.gx, sh.thr, sh.smem, st>>>(d, pl, sh.tile, ncomp, mode, p);
}
void launch_fft_x_inv(const Dev& d, const FftPlan1D& pl, int mode, const XinvParams& p, cudaStream_t st, int prec) {
    const bool f32 = prec != 0 && mode == 0;  // the grid-update chain (mode 1) stays FP64
    if (plan_pow2(pl)) f32 ? x_inv_rs<0, float2>(d, pl, mode, p, st) : x_inv_rs<0, double2>(d, pl, mode, p, st);
    else f32 ? x_inv_rs<1, float2>(d, pl, mode, p, st) : x_inv_rs<1, double2>(d, pl, mode, p, st);
}

// Time every candidate tile of the three tunable passes on this solve's grid (the solve's own
// state: the spectrum is scratch between iterations, and c0 / s0 are set) and keep the fastest.
// Candidates: every tile up to the model's upper bound that fits one block (fit_tile); each
// is launched once untimed and three times between CUDA events on the solve's stream.
template <class F>
static float time_launches(F&& launch, cudaStream_t st) {
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    launch();
    cudaEventRecord(a, st);
    for (int i = 0; i < 3; i++) launch();
    cudaEventRecord(b, st);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return ms;
}
static std::vector<int> tile_candidates(int T0) {
    std::vector<int> c;
    for (int t = 1; t <= T0; t++)
        if (t <= 8 || t == T0 || t % 4 == 0) c.push_back(t);
    return c;
}
template <int RS, class CT>
static void autotune_rs(const Dev& d, const FftPlan1D& pl1, const FftPlan1D& pl2, const FftPlan1D& pl3, const double* c0,
                        const double* s0, cudaStream_t st, std::vector<std::pair<TuneKey, int>>& found) {
    const int ct = sizeof(CT) == sizeof(float2) ? 1 : 0;
    const int nrows = d.n2 * d.n3, npairs = (nrows + 1) / 2;
    auto pick = [&](int pass, int T0, auto&& fits, auto&& launch) {
        if (tuned_tile(pass, RS, ct, d) > 0) return;
        int best = -1;
        float best_ms = 0.f;
        for (int t : tile_candidates(T0)) {
            int thr = 0;
            if (!fits(t, thr)) continue;
            const float ms = time_launches([&] { launch(t, thr); }, st);
            if (cudaGetLastError() != cudaSuccess) continue;
            if (best < 0 || ms < best_ms) {
                best = t;
                best_ms = ms;
            }
        }
        if (best > 0) found.push_back({TuneKey{pass, RS, ct, d.n1, d.n2, d.n3}, best});
    };
    const int mx_x = kernel_max_threads((const void*)k_fft_x_fwd<RS, CT>);
    pick(TUNE_XFWD, x_rows_per_block(d.n1),
         [&](int t, int& thr) {
             try { return fit_tile(t, 9, pl1, RS, 128, mx_x, thr) == t; } catch (std::exception&) { return false; }
         },
         [&](int t, int thr) {
             k_fft_x_fwd<RS, CT><<<(npairs + t - 1) / t, thr, (size_t)9 * t * d.n1 * sizeof(CT), st>>>(d, pl1, t, 0, OFF_SGAVG);
         });
    const int mx_y = std::min(kernel_max_threads((const void*)k_fft_y<true, RS, CT>), kernel_max_threads((const void*)k_fft_y<false, RS, CT>));
    pick(TUNE_Y, y_tile(d),
         [&](int t, int& thr) {
             try { return fit_tile(t, 1, pl2, RS, 64, mx_y, thr) == t; } catch (std::exception&) { return false; }
         },
         [&](int t, int thr) {
             k_fft_y<false, RS, CT><<<dim3((d.n1h + t - 1) / t, d.n3, 9), thr, (size_t)t * d.n2 * sizeof(CT), st>>>(d, pl2, t);
         });
    const int mx_z = kernel_max_threads((const void*)k_fft_z_green<RS, CT>);
    pick(TUNE_ZGREEN, z_tile(d),
         [&](int t, int& thr) {
             try { return fit_tile(t, 9, pl3, RS, 128, mx_z, thr) == t; } catch (std::exception&) { return false; }
         },
         [&](int t, int thr) {
             k_fft_z_green<RS, CT><<<dim3((d.n1h + t - 1) / t, d.n2), thr, (size_t)9 * t * d.n3 * sizeof(CT), st>>>(d, pl3, t, c0, s0);
         });
}

int fft_autotune(const Dev& d, const FftPlan1D& pl1, const FftPlan1D& pl2, const FftPlan1D& pl3, const double* c0,
                 const double* s0, int prec, cudaStream_t st) {
    const char* off = getenv("EVP_TUNE");  // EVP_TUNE=0: keep the model's tiles (for comparisons)
    if (off && off[0] == '0') return 0;
    std::vector<std::pair<TuneKey, int>> found;
    // each pass takes the radix set of its own axis (x forward: axis 1, y: axis 2, z: axis 3); tuning
    // both sets is cheap and covers whichever each axis needs
    for (int w = 0; w < (prec ? 2 : 1); w++) {
        if (w == 0) {
            autotune_rs<0, double2>(d, pl1, pl2, pl3, c0, s0, st, found);
            autotune_rs<1, double2>(d, pl1, pl2, pl3, c0, s0, st, found);
        } else {
            autotune_rs<0, float2>(d, pl1, pl2, pl3, c0, s0, st, found);
            autotune_rs<1, float2>(d, pl1, pl2, pl3, c0, s0, st, found);
        }
    }
    if (found.empty()) return 0;
    std::lock_guard<std::mutex> lk(g_tune_m);
    std::ofstream f;
    if (!g_tune_path.empty()) f.open(g_tune_path, std::ios::app);
    for (auto& kv : found) {
        if (g_tuned.count(kv.first)) continue;
        g_tuned[kv.first] = kv.second;
        const TuneKey& k = kv.first;
        if (f.is_open())
            f << "evp-tile " << k.pass << ' ' << k.rs << ' ' << k.ct << ' ' << k.n1 << ' ' << k.n2 << ' ' << k.n3 << ' '
              << kv.second << '\n';
    }
    return (int)found.size();
}

// ---------------------------------------------------------------- batched launches of the iteration's spectral passes
// As the voxel passes (evp_kernels.cu): each block finds its member in the launch's
// parameter and runs the member's body on its own block coordinates.
// A member takes part in the FP64 launch of a pass while its control block asks for FP64
// spectra and in the FP32 launch while it asks for FP32 (mixed precision).
template <class CT>
__device__ __forceinline__ bool batch_go(const IterCtl* c) {
    return c->active && ((c->prec != 0) == (sizeof(CT) == sizeof(float2)));
}
template <int RS, class CT>
__global__ void __launch_bounds__(256, 2) kb_fft_x_fwd(const __grid_constant__ BatchParams P) {
    const Job& jb = batch_job(P);
    const BatchSolve& m = P.E[jb.solve];
    if (!batch_go<CT>(m.ctl)) return;
    body_fft_x_fwd<RS, CT>(m.d, m.pl1, jb.tile, 0, m.ctl->sg_off, job_vb(jb));
}
template <bool INV, int RS, class CT>
__global__ void __launch_bounds__(256, 2) kb_fft_y(const __grid_constant__ BatchParams P) {
    const Job& jb = batch_job(P);
    const BatchSolve& m = P.E[jb.solve];
    if (!batch_go<CT>(m.ctl)) return;
    body_fft_y<INV, RS, CT>(m.d, m.pl2, jb.tile, job_vb(jb));
}
template <int RS, class CT>
__global__ void __launch_bounds__(256, 2) kb_fft_z_green(const __grid_constant__ BatchParams P) {
    const Job& jb = batch_job(P);
    const BatchSolve& m = P.E[jb.solve];
    if (!batch_go<CT>(m.ctl)) return;
    body_fft_z_green<RS, CT>(m.d, m.pl3, jb.tile, m.c0, m.s0, job_vb(jb));
}
template <int RS, class CT>
__global__ void __launch_bounds__(256, 2) kb_fft_x_inv(const __grid_constant__ BatchParams P) {
    __shared__ XinvParams xp;
    __shared__ int go;
    const Job& jb = batch_job(P);
    const BatchSolve& m = P.E[jb.solve];
    if (threadIdx.x == 0) {
        go = batch_go<CT>(m.ctl);
        xp = m.ctl->xinv;
    }
    __syncthreads();
    if (!go) return;
    body_fft_x_inv<RS, CT>(m.d, m.pl1, jb.tile, 9, 0, xp, job_vb(jb));
}

template <class CT>
static void member_fft_ct(const Dev& d, const FftPlan1D& pl1, const FftPlan1D& pl2, const FftPlan1D& pl3, int w,
                          MemberJobs& mj) {
    // the radix set of each pass follows its own axis, as in the single-solve launchers
    const int rs1 = plan_pow2(pl1) ? 0 : 1, rs2 = plan_pow2(pl2) ? 0 : 1, rs3 = plan_pow2(pl3) ? 0 : 1;
    auto put = [&](int k, const FftShape& sh, int rs) {
        mj.job[w][k] = Job{0, 0, sh.gx, sh.gy, sh.gz, sh.tile};
        mj.threads[w][k] = sh.thr;
        mj.smem[w][k] = sh.smem;
        mj.variant[w][k] = rs | (w << 1);
    };
    put(BK_XFWD, rs1 ? x_fwd_shape<1, CT>(d, pl1) : x_fwd_shape<0, CT>(d, pl1), rs1);
    const FftShape y = rs2 ? y_shape<1, CT>(d, pl2, 9) : y_shape<0, CT>(d, pl2, 9);
    put(BK_YFWD, y, rs2);
    put(BK_YINV, y, rs2);
    put(BK_ZGREEN, rs3 ? z_green_shape<1, CT>(d, pl3) : z_green_shape<0, CT>(d, pl3), rs3);
    put(BK_XINV, rs1 ? x_inv_shape<1, CT>(d, pl1, 9) : x_inv_shape<0, CT>(d, pl1, 9), rs1);
}

void member_jobs_fft(const Dev& d, const FftPlan1D& pl1, const FftPlan1D& pl2, const FftPlan1D& pl3, int prec, MemberJobs& mj) {
    member_fft_ct<double2>(d, pl1, pl2, pl3, 0, mj);
    if (prec) member_fft_ct<float2>(d, pl1, pl2, pl3, 1, mj);
    mj.has32 = prec != 0;
}

template <int RS, class CT>
static void batched_fft_ct(const BatchLaunch& L, const BatchParams& P, cudaStream_t st) {
    switch (L.kind) {
        case BK_XFWD: kb_fft_x_fwd<RS, CT><<<L.blocks, L.threads, L.smem, st>>>(P); break;
        case BK_YFWD: kb_fft_y<false, RS, CT><<<L.blocks, L.threads, L.smem, st>>>(P); break;
        case BK_ZGREEN: kb_fft_z_green<RS, CT><<<L.blocks, L.threads, L.smem, st>>>(P); break;
        case BK_YINV: kb_fft_y<true, RS, CT><<<L.blocks, L.threads, L.smem, st>>>(P); break;
        case BK_XINV: kb_fft_x_inv<RS, CT><<<L.blocks, L.threads, L.smem, st>>>(P); break;
        default: break;
    }
}
void launch_batched_fft(const BatchLaunch& L, const BatchParams& P, cudaStream_t st) {
    switch (L.variant) {
        case 0: batched_fft_ct<0, double2>(L, P, st); break;
        case 1: batched_fft_ct<1, double2>(L, P, st); break;
        case 2: batched_fft_ct<0, float2>(L, P, st); break;
        default: batched_fft_ct<1, float2>(L, P, st); break;
    }
}

// Raise the dynamic shared-memory limit of the FFT kernels (once per process).
template <int RS, class CT>
static void configure_ct() {
    const int lim = 160 * 1024;
    cudaFuncSetAttribute(k_fft_x_fwd<RS, CT>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    cudaFuncSetAttribute(k_fft_y<false, RS, CT>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    cudaFuncSetAttribute(k_fft_y<true, RS, CT>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    cudaFuncSetAttribute(k_fft_z_green<RS, CT>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    cudaFuncSetAttribute(k_fft_x_inv<RS, CT>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    cudaFuncSetAttribute(kb_fft_x_fwd<RS, CT>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    cudaFuncSetAttribute(kb_fft_y<false, RS, CT>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    cudaFuncSetAttribute(kb_fft_y<true, RS, CT>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    cudaFuncSetAttribute(kb_fft_z_green<RS, CT>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    cudaFuncSetAttribute(kb_fft_x_inv<RS, CT>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
}
template <int RS>
static void configure_rs() {
    const int lim = 160 * 1024;
    configure_ct<RS, double2>();
    configure_ct<RS, float2>();
    cudaFuncSetAttribute(k_fft_z_integ<RS>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    cudaFuncSetAttribute(k_green_x_fwd<RS>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    cudaFuncSetAttribute(k_green_x_inv<RS>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
}
void fft_configure() {
    configure_rs<0>();
    configure_rs<1>();
}

}  // namespace evp
