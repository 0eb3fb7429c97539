// evp_green.cu -- operator-level C ABI: the spectral Green-operator application.
//
// evp_green_apply applies the periodic Green operator of a homogeneous
// reference medium to a 9-component polarization field held in device memory
// (convolution_with_Goper with form_G for igamma = 0, various_functions.f90:640-809
// and 966-1059): forward 3-D DFT, Gamma(xi):tau(xi) with the DC term zeroed and
// -s0 on Nyquist planes, inverse DFT, real part / N.  It is the inner
// operator of every equilibrium iteration of the solver, exposed for callers
// that drive their own fixed-point scheme.
#include "../../include/evp.h"
#include "evp_dev.cuh"

#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>
#include <vector>

namespace evp {
void set_last_error(const std::string& m);

static void host_twiddles(int n, double2* out) {
    for (int e = 0; e < n; e++) {
        long double ang = -2.0L * 3.14159265358979323846264338327950288L * (long double)e / (long double)n;
        out[e] = make_double2((double)cosl(ang), (double)sinl(ang));
    }
}

static void configure_once() {
    static std::once_flag flag;
    std::call_once(flag, [] { fft_configure(); });
}

static int check_args(const double* d_tau, double* d_out, int n1, int n2, int n3, const double* c0, const double* s0) {
    if (!d_tau || !d_out || !c0 || !s0) { set_last_error("evp_green_apply: null argument"); return -7; }
    if (n1 < 1 || n2 < 1 || n3 < 1) { set_last_error("evp_green_apply: grid dimensions must be positive"); return -7; }
    return 0;
}

}  // namespace evp

extern "C" int evp_green_apply(const double* d_tau, double* d_out, int n1, int n2, int n3, const double* c0, const double* s0,
                               void* stream) {
    using namespace evp;
    int rc = check_args(d_tau, d_out, n1, n2, n3, c0, s0);
    if (rc) return rc;
    FftPlan1D pl1, pl2, pl3;
    try {
        pl1 = make_plan(n1); pl2 = make_plan(n2); pl3 = make_plan(n3);
    } catch (std::exception& e) {
        set_last_error(e.what());
        return -2;
    }
    configure_once();
    cudaStream_t st = (cudaStream_t)stream;
    Dev d{};
    d.n1 = n1; d.n2 = n2; d.n3 = n3;
    d.n1h = n1 / 2 + 1;
    d.N = (long long)n1 * n2 * n3;
    const size_t nspec = 9 * (size_t)d.n1h * n2 * n3;
    std::vector<double2> tw(n1 + n2 + n3);
    host_twiddles(n1, tw.data());
    host_twiddles(n2, tw.data() + n1);
    host_twiddles(n3, tw.data() + n1 + n2);
    double2 *spec = nullptr, *dtw = nullptr;
    double* cs = nullptr;
    int* err = nullptr;
    auto cleanup = [&]() {
        cudaFree(spec); cudaFree(dtw); cudaFree(cs); cudaFree(err);
    };
    if (cudaMalloc(&spec, nspec * sizeof(double2)) != cudaSuccess || cudaMalloc(&dtw, tw.size() * sizeof(double2)) != cudaSuccess ||
        cudaMalloc(&cs, 162 * sizeof(double)) != cudaSuccess || cudaMalloc(&err, sizeof(int)) != cudaSuccess) {
        cleanup();
        set_last_error("evp_green_apply: device allocation failed");
        return -6;
    }
    cudaMemcpyAsync(dtw, tw.data(), tw.size() * sizeof(double2), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(cs, c0, 81 * sizeof(double), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(cs + 81, s0, 81 * sizeof(double), cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(err, 0, sizeof(int), st);
    d.spec = spec;
    d.tw1 = dtw; d.tw2 = dtw + n1; d.tw3 = dtw + n1 + n2;
    d.err = err;
    launch_green_apply(d, pl1, pl2, pl3, d_tau, d_out, cs, cs + 81, st);
    int herr = 0;
    cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaError_t ce = cudaStreamSynchronize(st);
    cleanup();
    if (ce != cudaSuccess) {
        set_last_error(std::string("evp_green_apply: ") + cudaGetErrorString(ce));
        return -6;
    }
    if (herr) {
        set_last_error("evp_green_apply: singular acoustic tensor");
        return -3;
    }
    return 0;
}
