// evp_control.cu -- the serial tail of one equilibrium iteration, on the device.
//
// After the iteration kernels of an increment have run, the reference's driver
// forms the macroscopic averages, updates the mixed boundary conditions
// (calc_velgradavg_corr + state_6x6_evpsc, various_functions.f90:1526-1705),
// normalises the error norms, picks the next mixing factor and decides whether
// the increment has converged (LS-EVPFFT.f90:277-430).  k_control does exactly
// that, one thread per solve, on the sums the kernels left in the solve's result
// buffer, so that the next iteration can be launched without the host in the
// loop (and many iterations, of many solves, captured in one CUDA graph).  This
// file is compiled with -fmad=false: the tail's arithmetic keeps the plain
// multiply-then-add rounding of the reference's serial code.  Decisions that need
// the host (the ictrl = -1 sub-stepping check, which launches a kernel and may
// roll the increment back) end the solve's iteration with EV_HOST.
#include "evp_dev.cuh"
#include "evp_math.cuh"

namespace evp {

// state_6x6_evpsc (various_functions.f90:1638-1705): the VPSC-Voigt macroscopic state with mixed
// strain-rate / stress components.  The system matrix and its LU factors are per-increment
// constants (state_6x6_factor, on the host); here the right-hand side and the substitution.
__device__ void state_6x6_dev(const IterCtl& c, double* dbar, double* sbar, const double* devp0, double* scauchy,
                              double* dsim) {
    double profac[6], dbarv[6], sbarv[6], devp0v[6], aux6[6], aux6a[6], a33[9];
    for (int i = 1; i <= 6; i++) profac[i - 1] = 1.0 + (i / 4);
    for (int i = 0; i < 6; i++) {
        dbarv[i] = dsim[3 * ijv_a(i) + ijv_b(i)];
        sbarv[i] = scauchy[3 * ijv_a(i) + ijv_b(i)];
    }
    b6_to_t2(devp0, a33);
    for (int i = 0; i < 6; i++) devp0v[i] = a33[3 * ijv_a(i) + ijv_b(i)];
    for (int i = 0; i < 6; i++) aux6[i] = dbarv[i] - devp0v[i];
    for (int i = 0; i < 6; i++) {
        aux6a[i] = -1.0 * c.idsim[i] * aux6[i];
        for (int j = 0; j < 6; j++) aux6a[i] = aux6a[i] + c.xmv[6 * i + j] * c.iscau[j] * sbarv[j] * profac[j];
    }
    lu_solve(c.lu, 6, c.piv, aux6a);
    for (int i = 0; i < 6; i++) {
        aux6[i] = c.idsim[i] * aux6[i] + c.iscau[i] * aux6a[i];
        sbarv[i] = c.iscau[i] * sbarv[i] + c.idsim[i] * aux6a[i];
    }
    for (int i = 0; i < 6; i++) dbarv[i] = aux6[i] + devp0v[i];
    for (int i = 0; i < 6; i++) {
        dsim[3 * ijv_a(i) + ijv_b(i)] = dbarv[i];
        dsim[3 * ijv_b(i) + ijv_a(i)] = dbarv[i];
        scauchy[3 * ijv_a(i) + ijv_b(i)] = sbarv[i];
        scauchy[3 * ijv_b(i) + ijv_a(i)] = sbarv[i];
    }
    t2_to_b6(dsim, dbar);
    t2_to_b6(scauchy, sbar);
}

// calc_velgradavg_corr tail (various_functions.f90:1575-1631) on the solid stress sum.
__device__ void velgradavg_corr_dev(IterCtl& c, const double* sgsol6) {
    s6_to_t2(sgsol6, c.sgavg);
    for (int k = 0; k < 9; k++) c.sgavgsol[k] = c.sgavg[k] / c.wphcsol;
    c.svmavg = vm_stress(c.sgavg);
    double a33[9];
    for (int i = 0; i < 6; i++) {
        const int ii = ijv_a(i), jj = ijv_b(i);
        a33[3 * ii + jj] = c.iscau[i] * (c.scauchy[3 * ii + jj] - c.sgavg[3 * ii + jj]);
        a33[3 * jj + ii] = c.iscau[i] * (c.scauchy[3 * jj + ii] - c.sgavg[3 * jj + ii]);
    }
    c.errsbc = frob3(a33);
    double vsym[9], vasym[9], dbar[6], sbar[6], devp0[6];
    sym33(c.velgradavg, vsym);
    antisym33(c.velgradavg, vasym);
    t2_to_b6(vsym, dbar);
    t2_to_b6(c.sgavg, sbar);
    for (int i = 0; i < 6; i++) {
        double s = 0.0;
        for (int j = 0; j < 6; j++) s += c.mev[6 * i + j] * sbar[j];
        devp0[i] = dbar[i] - s;
    }
    state_6x6_dev(c, dbar, sbar, devp0, c.scauchy, c.dsim);
    double w[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int ii = 0; ii < 3; ii++)
        for (int jj = 0; jj < 3; jj++) {
            if (ii == jj) {
                w[3 * ii + jj] = 0.0;
                continue;
            }
            const int a = c.iudot[3 * ii + jj], b = c.iudot[3 * jj + ii];
            if (a == 1 && b == 0) {
                w[3 * ii + jj] = c.udot[3 * ii + jj] - c.dsim[3 * ii + jj];
                w[3 * jj + ii] = -w[3 * ii + jj];
            } else if (a == 0 && b == 1) {
            } else if (a == 1 && b == 1) {
                w[3 * ii + jj] = 0.5 * (c.udot[3 * ii + jj] - c.udot[3 * jj + ii]);
            } else {
                w[3 * jj + ii] = 0.0;
            }
        }
    for (int k = 0; k < 9; k++) c.xinv.dvelgradavg[k] = (c.dsim[k] - vsym[k]) + (w[k] - vasym[k]);
}

__device__ void stop(IterCtl& c, int event, int bits) {
    c.event = event;
    c.errbits |= bits;
    c.active = 0;
}

// One equilibrium iteration's tail for one solve: the host loop of LS-EVPFFT.f90:233-430
// between the kernels of one iteration and the launch of the next.
__device__ void control_one(IterCtl& c, const double* red, int err) {
    c.iter++;
    c.total_iters++;
    // the device error word first (singular voxel operator, non-finite Newton result, form_G failure)
    if (err & 1) return stop(c, -3, 1);
    if (err & 2) return stop(c, -4, 2);
    if (err & 4) return stop(c, -3, 4);
    if (err & 8) return stop(c, -6, 64);
    const double* cr = red + OFF_CORR;
    for (int k = 0; k < 9; k++) {
        c.velgradavg[k] = cr[k];
        c.velgradavggas[k] = cr[9 + k];
        c.velgradavgsol[k] = cr[18 + k];
    }
    if (c.wphcgas > 0.0)
        for (int k = 0; k < 9; k++) c.velgradavggas[k] /= c.wphcgas;
    for (int k = 0; k < 9; k++) c.velgradavgsol[k] /= c.wphcsol;
    if (!c.kinematic) {  // mixing factor of the next iteration (LS-EVPFFT.f90:277-311)
        const double dls = cr[28] > 0.0 ? sqrt(cr[27] / cr[28]) : 0.0;
        const double dlg = cr[30] > 0.0 ? sqrt(cr[29] / cr[30]) : 0.0;
        const double dl = fmax(dls, dlg);
        c.corr.mix = fmax(1.0e-8, fmin(1.0, 5.0e-2 / fmax(dl, 5.0e-2)));
    }
    const double* nw = red + OFF_NEWTON;
    double errs = nw[0], erre = nw[1];
    if (erre < 0 || errs < 0) return stop(c, -4, 8);
    erre = sqrt(erre);
    errs = sqrt(errs);
    velgradavg_corr_dev(c, nw + 2);
    c.erre = erre / c.lvmavg;
    c.errs = errs / c.svmavg;
    c.errsbc = c.errsbc / c.svmavg;
    c.fresh = 0;
    c.sg_off = OFF_NEWTON + 8;
    if (c.ictrl == 0) {  // von Mises strain-rate control: tdot from the imposed increment
        double vs[9];
        sym33(c.velgradavg, vs);
        c.tdot = c.devmapp / vm_strain(vs);
        c.tdotref = c.tdot;
        c.newton.tdot = c.tdot;
    }
    const bool conv = c.errs <= c.error && c.erre <= c.error && c.errsbc <= c.error;
    c.did_converge = conv ? 1 : 0;
    if (c.prec != 0 && !conv) {  // FP32 iterations stagnating above the tolerance: FP64 from here on
        c.hist[c.nhist & 3] = fmax(c.errs, fmax(c.erre, c.errsbc));
        c.nhist++;
        if (c.nhist >= 4 && c.hist[(c.nhist - 1) & 3] > 0.7 * c.hist[(c.nhist - 4) & 3]) c.prec = 0;
    }
    int ev = EV_RUNNING;
    if (c.ictrl == -1) {
        if (c.tdot > c.tdotmin) {
            if (conv || c.iter == c.itmax) ev = EV_HOST;
        } else if (c.iter == c.itmax) {
            ev = EV_ACCEPTED;
        }
    }
    if (ev == EV_RUNNING && conv) ev = EV_CONVERGED;
    if (ev == EV_RUNNING && c.iter >= 100000) return stop(c, -4, 32);
    if (ev != EV_RUNNING) {
        c.event = ev;
        c.active = 0;
    }
}

// One warp per solve: the warp copies the solve's control block and the sums it reads into
// shared memory (coalesced), lane 0 does the serial tail there, and the warp writes the block
// back; the serial code then waits on shared memory instead of one global load after another.
constexpr int kCtlWords = (int)(sizeof(IterCtl) / 8);
static_assert(sizeof(IterCtl) % 8 == 0, "IterCtl is copied in 8-byte words");

__global__ void __launch_bounds__(32) k_control(const BatchSolve* __restrict__ E, int n, int* __restrict__ events) {
    const int i = blockIdx.x;
    if (i >= n) return;
    __shared__ IterCtl c;
    __shared__ double red[OFF_NEWTON + 14];
    __shared__ int err;
    IterCtl* g = E[i].ctl;
    unsigned long long* cw = reinterpret_cast<unsigned long long*>(&c);
    const unsigned long long* gw = reinterpret_cast<const unsigned long long*>(g);
    for (int w = threadIdx.x; w < kCtlWords; w += 32) cw[w] = gw[w];
    const double* r = E[i].d.red;
    for (int k = OFF_CORR + threadIdx.x; k < OFF_NEWTON + 14; k += 32) red[k] = r[k];
    if (threadIdx.x == 0) err = *(volatile int*)E[i].d.err;
    __syncwarp();
    const bool run = c.active != 0;
    if (run && threadIdx.x == 0) control_one(c, red, err);
    __syncwarp();
    if (run) {
        unsigned long long* gwo = reinterpret_cast<unsigned long long*>(g);
        for (int w = threadIdx.x; w < kCtlWords; w += 32) gwo[w] = cw[w];
    }
    if (threadIdx.x == 0) events[i] = c.active ? EV_RUNNING : c.event;
}

void launch_control(const BatchSolve* E, int n, int* events, cudaStream_t st) {
    k_control<<<n, 32, 0, st>>>(E, n, events);
}

}  // namespace evp
