// evp_dev.cuh -- device-resident state of one LS-EVPFFT solve and kernel entry points.
//
// HBM layout: structure of arrays, FP64, one contiguous array per field with
// the component index outermost: field[c * N + v], voxel v = i + n1*(j + n2*k).
// Symmetric tensors are stored as s6 = (11,22,33,23,13,12); full 3x3 tensors
// row-major (c = 3*row + col); 6x6 operators row-major (c = 6*row + col).
// The half spectrum of the FFT work array is complex128
// spec[c][k][j][kx], kx in [0, n1/2].
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <string>

namespace evp {

constexpr int kMaxSysDev = 24;

// Per-phase constants (phase_type, types.f90:96-118) in device memory.
struct PhaseDev {
    int nsyst, nmodes, igas, int_exp;  // int_exp: every nrs-1 is an integer in [0,64]
    int nsm[3];
    double nrs[kMaxSysDev], gamd0[kMaxSysDev], hpfac[kMaxSysDev];
    double tau0f[kMaxSysDev], tau0b[kMaxSysDev];
    double tau1[3], thet0[3], thet1[3];  // per mode, from its last system (harden, various_functions.f90:1466-1470)
    double hard[kMaxSysDev * kMaxSysDev];
    double dnca[kMaxSysDev * 3], dbca[kMaxSysDev * 3];
    double C[81];
};

// Offsets (in doubles) of the per-kernel results in the small result buffer.
enum : int {
    OFF_SGAVG = 0,    // 6   sum wgtc*sg over all voxels
    OFF_DU = 8,       // 9   BC correction of the average velgrad (reference config)
    OFF_CORR = 24,    // 31  sum velgrad*wgtc (all, gas, solid), dL mixing sums
    OFF_NEWTON = 64,  // 14  errs, erre, sum wgtc*sg (solid), sum wgtc*sg (all)
    OFF_INIT = 80,    // 36  sum cg66*wgtc (solid)
    OFF_UPD1 = 120,   // 40  F averages, weights, max solid vm rate
    OFF_DU2 = 160,    // 9   average-velgrad fix of update_tensor_config
    OFF_UPD3 = 176,   // 30+13 averages, hardening sums, last solid voxel
    OFF_DIAG = 224,   // 24+ diagnostics reductions
    OFF_C0 = 272,     // 72 macro tangent sums (b-basis dsg/de, PK1 tangent)
    OFF_KIN = 392,    // 4   kinematic increment maxima
    OFF_DISP = 344,   // 30  init_defgrad sums (F^-1 w J all/solid/gas, w J solid/gas, J w)
    OFF_DC = 400,     // 18  DC of the grid-update spectrum (complex x 9)
    OFF_G0 = 420,     // 81  real-space Green operator at the origin
    RED_OUT_SIZE = 512
};

enum : int { CNT_SGAVG = 0, CNT_XINV, CNT_CORR, CNT_NEWTON, CNT_INIT, CNT_UPD1, CNT_UPD2, CNT_UPD3, CNT_DIAG, CNT_DIAG2, CNT_C0, CNT_KIN, CNT_G0, CNT_DISP, CNT_N };

// Block coordinates of a kernel body: the hardware block index for a launch over one
// solve, or the solve-local block index that a batched launch decodes from its job
// table (nx: the solve-local grid extent along x, which is the whole grid of a 1-D launch).
struct VB {
    int x, y, z, nx;
};
#ifdef __CUDACC__
__device__ __forceinline__ VB hw_vb() { return VB{(int)blockIdx.x, (int)blockIdx.y, (int)blockIdx.z, (int)gridDim.x}; }
#endif

struct FftPlan1D {
    int n;
    int nst;
    int rad[8];
};

struct Dev {
    long long N;
    int n1, n2, n3, n1h, n3node;
    int nsys;  // max nsyst over phases (array stride of the per-system fields)
    int grid;  // blocks of the voxel kernels
    double wgt;
    // voxel state
    double *sg, *sgt, *edotp, *ept, *disgradsym;         // s6
    double *velgrad, *velgradold, *dvr;                  // 9
    double *F, *Finv, *Fe, *Fp, *Finc, *Feinc, *ag;      // 9
    double *detF, *wgtc, *epvm, *gacumgr;                // 1
    double *sg66, *c066mod, *cG, *cgas;                  // 36 (cG, cgas may be null)
    double *c066inv;                                     // 36: inverse of c066mod, formed with it
    double *sch;                                         // 5*nsys   [(s*5+c)*N + v]
    double *crss, *trialtau;                             // 2*nsys   [(s*2+c)*N + v]
    double *gamdot;                                      // nsys
    double *eth;                                         // 9 or null
    uint8_t *gas, *phase;                                // phase index 0-based
    // snapshot copies (take_snapshot / rollback)
    double *s_velgrad, *s_velgradold, *s_sg, *s_edotp, *s_gamdot, *s_trialtau;
    // spectrum, twiddles, grid-update scratch
    double2 *spec;
    double2 *tw1, *tw2, *tw3;
    float2 *tw1f, *tw2f, *tw3f;  // FP32 twiddles of the mixed-precision path (may be null)
    double *dv3, *xnode;
    // tabulated Green operator of IGAMMA 1 and 2: 81 components per half-spectrum point,
    // goper[c * (n1h n2 n3) + (k3 n2 + j) n1h + kx]; gtab = 1 while the current process uses it
    double* goper;
    int gtab;
    double* Fini;  // initial deformation gradient (IDISPINI 1, 2 only; null: identity)
    // reductions
    double *partials, *red;
    // Newton activity counters (null unless the solve is profiled): [0] warp passes of the
    // evaluation loop, [1] voxel evaluations done in them, [2] Newton steps, [3] hardening
    // updates, [4] voxels, [5] warp passes of the Newton-step loop
    unsigned long long* nstats;
    unsigned int *counters;
    int *err;  // error word: bit 0 singular matrix, bit 1 non-finite Newton result, bit 2 form_G failure,
               // bit 3 a TMA bulk copy that did not complete within its bounded wait
    const PhaseDev *ph;
    int nph;
};

struct CorrParams {
    double mix, Lscale;
    int do_mix, kinematic;
};
struct NewtonParams {
    double tdot, error, erroral, complgas;
    int modal, thermo, iuphard;
};
struct XinvParams {
    double dvelgradavg[9];
    double dinv[9];  // inverse of the average F^{-1} (current config)
};
struct Upd1Params {
    double tdot;
    int iupdate;
};
struct Upd2Params {
    double velgradavg[9];
};
struct Upd3Params {
    double tdot;
    int iupdate, iuphard;
    long long vlast;  // last solid voxel in loop order (for the eelav quirk, LS-EVPFFT.f90:482-483)
};

// Control block of one solve's equilibrium iteration, in device memory.  The host
// fills it at the start of an increment (and after a sub-step restart); the
// iteration kernels read their parameters from it; k_control, run after every
// iteration, does the serial tail of the reference's loop on the device (the
// averages and the boundary-condition update of calc_velgradavg_corr and
// state_6x6_evpsc, the error norms, the mixing factor, the convergence test and
// the time-step rules, LS-EVPFFT.f90:277-430) and stops the solve's iteration
// with an event code the host reads, so that no iteration waits for the host.
enum : int { EV_RUNNING = 0, EV_CONVERGED = 1, EV_ACCEPTED = 2, EV_HOST = 3 };
struct IterCtl {
    // read by the iteration kernels
    int active;  // 1 while this solve iterates; 0 once k_control has set an event
    int prec;    // spectrum precision of the next iteration: 0 FP64, 1 FP32
    int fresh;   // the next iteration is the first of its increment: form the stress average first
    int sg_off;  // where the PK1 prologue reads the average stress (OFF_SGAVG or OFF_NEWTON + 8)
    CorrParams corr;
    XinvParams xinv;
    NewtonParams newton;
    // iteration state
    int iter, itmax, ictrl, event;  // event: EV_* or a negative status code
    int errbits, kinematic, did_converge, nhist;
    long long total_iters;
    double error, tdotmin, devmapp, lvmavg;
    double erre, errs, errsbc, svmavg, wphcsol, wphcgas;
    double hist[4];  // the last four error maxima of the FP32 iterations (ring)
    double velgradavg[9], velgradavggas[9], velgradavgsol[9], sgavg[9], sgavgsol[9];
    // per-increment constants of calc_velgradavg_corr / state_6x6_evpsc, formed on the host at the
    // start of the increment: de_ds in the b-basis (mev), its Voigt form (xmv) and the LU factors
    // and pivots of the mixed-BC system (they depend only on de_ds and the process's masks)
    double mev[36], xmv[36], lu[36];
    int piv[6], pad6[2];
    // boundary conditions of the current process (dsim and scauchy change every iteration)
    int iscau[6], idsim[6], iudot[9];
    double udot[9], dsim[9], scauchy[9];
    double tdot, tdotref;
};

// One member of a batched launch: the solve's device state, its FFT plans, its
// control block and its reference-medium stiffness / compliance (device arrays).
struct BatchSolve {
    Dev d;
    FftPlan1D pl1, pl2, pl3;
    IterCtl* ctl;
    const double* c0;
    const double* s0;
};
// A batched launch covers, for every member it serves, the blocks
// [blk0, blk0 + gx * gy * gz) of the launch; inside them the member's kernel body
// sees the solve-local block (b % gx, (b / gx) % gy, b / (gx gy)), exactly the
// grid and tile its own single-solve launch would use.
struct Job {
    int solve, blk0, gx, gy, gz, tile;
};
// The passes of one equilibrium iteration, in launch order (the stress average that the first
// iteration of an increment starts from is formed when the increment's iterations start).
enum BatchKind : int { BK_XFWD, BK_YFWD, BK_ZGREEN, BK_YINV, BK_XINV, BK_CORR, BK_NEWTON, BK_N };
struct BatchLaunch {
    int kind, variant;  // variant: FFT passes rs | (FP32 << 1); Newton: the kernel (newton_variant)
    int job0, njobs;    // slice of the plan's job table
    int blocks, threads;
    size_t smem;
};
// The members of one batched launch travel as its kernel parameter (a __grid_constant__
// struct in the constant bank: read-only and uniform, so the bodies' loads of sizes and
// pointers are as cheap as a single-solve launch's).  Up to kBatchChunk members per launch
// (26.6 kB of the 32 kB parameter space); larger batches take several launches per pass.
constexpr int kBatchChunk = 40;
struct BatchParams {
    int njobs, pad;
    Job jobs[kBatchChunk];  // job.solve indexes E
    BatchSolve E[kBatchChunk];
};
// Job-table entries of one member for every pass it takes part in (host side of the batch
// plan): [0] the FP64 launch shape of each pass, [1] the FP32 one of the spectral passes of a
// mixed-precision member (has32).
struct MemberJobs {
    Job job[2][BK_N];
    int variant[2][BK_N];
    int threads[2][BK_N];
    size_t smem[2][BK_N];
    bool has32;
};

#ifdef __CUDACC__
// Block side of a batched launch: the job (member) covering this block (binary search on
// blk0) and the solve-local block coordinates inside it.
__device__ __forceinline__ const Job& batch_job(const BatchParams& P) {
    int lo = 0, hi = P.njobs - 1;
    const int b = blockIdx.x;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (P.jobs[mid].blk0 <= b) lo = mid;
        else hi = mid - 1;
    }
    return P.jobs[lo];
}
__device__ __forceinline__ VB job_vb(const Job& jb) {
    const int l = (int)blockIdx.x - jb.blk0;
    return VB{l % jb.gx, (l / jb.gx) % jb.gy, l / (jb.gx * jb.gy), jb.gx};
}
// Sum of field f of nblk block partials (partials[f * nblk + b]) by one warp: lane l adds
// blocks l, l + 32, ... in order, then a fixed shuffle tree; the result is in lane 0.
// The loads go out eight at a time (one L2 round trip per eight blocks instead of per block);
// the additions keep the one-block-at-a-time order.
__device__ __forceinline__ double fold_sum(const double* partials, int nblk, int f, int lane) {
    const double* q = partials + (size_t)f * nblk;
    double s = 0.0;
    int b = lane;
    for (; b + 7 * 32 < nblk; b += 8 * 32) {
        double x[8];
#pragma unroll
        for (int i = 0; i < 8; i++) x[i] = __ldcg(q + b + 32 * i);
#pragma unroll
        for (int i = 0; i < 8; i++) s += x[i];
    }
    for (; b < nblk; b += 32) s += __ldcg(q + b);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    return s;  // in lane 0
}
#endif

// ---- launch wrappers (stream-ordered)
// keepF: F, F^-1, det F and the unscaled weights w J were set by launch_dispini; the weights
// are divided by detFavg here (IO_functions.f90:934) and weight the start-up tangent sum
void launch_init(const Dev& d, const double* euler, const int* grain, const double* hp, const double* udot9, const double* u6t,
                 int keepF, double detFavg, cudaStream_t st);
// init_defgrad per voxel (IO_functions.f90:893-921): F = grad(u) + diag(delt) from the gradient
// field (component 3m + l = d u_l / d x_m), F_ini = F, det F, F^-1, w J and the OFF_DISP sums
void launch_dispini(const Dev& d, const double* grad, double delt, cudaStream_t st);
void launch_sgavg(const Dev& d, cudaStream_t st);
void launch_prologue(const Dev& d, const double* c0, const double* goperr0, int do_schmid, int modal, cudaStream_t st);
void launch_goperr0(const Dev& d, const double* c0, const double* s0, int igamma, cudaStream_t st);
// form_G for IGAMMA 1 and 2: tabulate the Green operator at every half-spectrum point
void launch_goper_tab(const Dev& d, const double* c0, const double* s0, int igamma, cudaStream_t st);
void launch_gas_compl(const Dev& d, double tdot, double complgas, int modal, cudaStream_t st);
void launch_corr(const Dev& d, const CorrParams& p, cudaStream_t st);
void launch_newton(const Dev& d, const NewtonParams& p, cudaStream_t st);
void launch_upd1(const Dev& d, const Upd1Params& p, cudaStream_t st);
void launch_upd2(const Dev& d, const Upd2Params& p, cudaStream_t st);
void launch_upd3(const Dev& d, const Upd3Params& p, cudaStream_t st);
void launch_diag(const Dev& d, double Lfloor, cudaStream_t st);
void launch_c0(const Dev& d, double tdot, double tdotref, cudaStream_t st);
void launch_kinematic(const Dev& d, double tdot_step, cudaStream_t st);
void launch_cell2node(const Dev& d, double tdot, int ideriv, cudaStream_t st);

// Batched equilibrium iteration: the member's per-pass launch shape (its single-solve grid
// and tile) and the launches over a job table (E, jobs: device arrays).
void member_jobs_voxel(const Dev& d, int modal, MemberJobs& mj);
void member_jobs_fft(const Dev& d, const FftPlan1D& pl1, const FftPlan1D& pl2, const FftPlan1D& pl3, int prec, MemberJobs& mj);
void launch_batched_voxel(const BatchLaunch& L, const BatchParams& P, cudaStream_t st);
void launch_batched_fft(const BatchLaunch& L, const BatchParams& P, cudaStream_t st);
// the serial tail of one iteration for n solves (evp_control.cu); events[i] = EV_* or a status code
void launch_control(const BatchSolve* E, int n, int* events, cudaStream_t st);

// Measured tile choice of the spectral passes (evp_fft.cu): the cache file (empty: none) and
// the timing of the candidates for a solve's grid at open (returns how many pass shapes were
// tuned; 0 when the process or the file knew them all).
void fft_tune_cache(const std::string& path);
int fft_autotune(const Dev& d, const FftPlan1D& pl1, const FftPlan1D& pl2, const FftPlan1D& pl3, const double* c0,
                 const double* s0, int prec, cudaStream_t st);

// FFT engine (evp_fft.cu)
FftPlan1D make_plan(int n);
// prec 1: the equilibrium chain's spectrum, FFTs and Green operator in FP32 (mixed precision)
void launch_fft_x_fwd(const Dev& d, const FftPlan1D& pl, int mode, int sg_off, cudaStream_t st, int prec = 0);
void fft_configure();
// Green operator applied to 9 real fields tau -> out (caller-owned device arrays);
// d supplies the grid, spectrum scratch, twiddles and error word.
void launch_green_apply(const Dev& d, const FftPlan1D& pl1, const FftPlan1D& pl2, const FftPlan1D& pl3, const double* tau,
                        double* out, const double* c0, const double* s0, cudaStream_t st);
void launch_fft_y(const Dev& d, const FftPlan1D& pl, int ncomp, bool inverse, cudaStream_t st, int prec = 0);
void launch_fft_z_green(const Dev& d, const FftPlan1D& pl, const double* c0, const double* s0, cudaStream_t st, int prec = 0);
void launch_fft_z_integ(const Dev& d, const FftPlan1D& pl, int ideriv, cudaStream_t st);
// gradient_tensor1 (various_functions.f90:56-112) of a vector field given as 9 real fields with
// component 3m + l = u_l: out component 3m + l = d u_l / d x_m (spectral derivative ideriv)
void launch_gradient(const Dev& d, const FftPlan1D& pl1, const FftPlan1D& pl2, const FftPlan1D& pl3, const double* u9,
                     double* out, int ideriv, cudaStream_t st);
void launch_fft_x_inv(const Dev& d, const FftPlan1D& pl, int mode, const XinvParams& p, cudaStream_t st, int prec = 0);

}  // namespace evp
