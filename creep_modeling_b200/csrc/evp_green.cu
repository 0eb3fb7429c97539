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

// ---------------------------------------------------------------- allocation-free variant
// Some callers cannot call cudaMalloc: a host application whose device memory
// is already owned by another allocator (a pre-reserved pool such as PyTorch's
// caching allocator, or a serving loop that has handed its whole HBM budget to
// admitted solves), or a latency-critical loop that cannot afford the
// device-wide synchronization that cudaMalloc/cudaFree imply.  For them,
// evp_green_apply_noalloc keeps its scratch (half spectrum, twiddles, c0/s0
// and the error word) in the fixed file-scope array below.  Every GPU that
// loads this library holds the array (about 2.5 MB) until the process exits;
// all calls on a device share it, so calls whose device work overlaps (for
// example on two streams) race and must be serialized by the caller.
namespace evp {
constexpr size_t kNoAllocMaxHalfVox = 17408;  // max (n1/2+1)*n2*n3, e.g. a 32^3 grid
constexpr int kNoAllocMaxEdge = 256;          // max n1, n2, n3 (twiddle slots)
constexpr size_t kNoAllocSpec = 9 * kNoAllocMaxHalfVox;
constexpr size_t kNoAllocTw = kNoAllocSpec;                  // offset of the twiddles (3 x 256)
constexpr size_t kNoAllocCs = kNoAllocTw + 3 * kNoAllocMaxEdge;  // offset of c0, s0 (162 doubles)
constexpr size_t kNoAllocErr = kNoAllocCs + 81;              // offset of the error word
constexpr size_t kNoAllocTotal = kNoAllocErr + 1;
}  // namespace evp

static __device__ __align__(256) double2 g_green_scratch[evp::kNoAllocTotal];

namespace evp {
constexpr int kMaxDevices = 64;
static double2* g_scratch_addr[kMaxDevices] = {};
static std::mutex g_scratch_mu;

// Device address of g_green_scratch for the current device.  The first call on
// a device resolves it with cudaGetSymbolAddress (with that device current).
static int noalloc_scratch(double2** out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        set_last_error("evp_green_apply_noalloc: no current CUDA device");
        return -6;
    }
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
        double2* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress((void**)&p, g_green_scratch);
        if (e != cudaSuccess || !p) {
            set_last_error(std::string("evp_green_apply_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
            return -6;
        }
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return 0;
}
}  // namespace evp

extern "C" int evp_green_apply_noalloc(const double* d_tau, double* d_out, int n1, int n2, int n3, const double* c0,
                                       const double* s0, void* stream) {
    using namespace evp;
    int rc = check_args(d_tau, d_out, n1, n2, n3, c0, s0);
    if (rc) return rc;
    const size_t halfvox = (size_t)(n1 / 2 + 1) * n2 * n3;
    if (halfvox > kNoAllocMaxHalfVox || n1 > kNoAllocMaxEdge || n2 > kNoAllocMaxEdge || n3 > kNoAllocMaxEdge) {
        set_last_error("evp_green_apply_noalloc: grid " + std::to_string(n1) + "x" + std::to_string(n2) + "x" +
                       std::to_string(n3) + " exceeds the fixed scratch ((n1/2+1)*n2*n3 <= " +
                       std::to_string(kNoAllocMaxHalfVox) + ", every edge <= " + std::to_string(kNoAllocMaxEdge) +
                       "); use evp_green_apply");
        return -7;
    }
    FftPlan1D pl1, pl2, pl3;
    try {
        pl1 = make_plan(n1); pl2 = make_plan(n2); pl3 = make_plan(n3);
    } catch (std::exception& e) {
        set_last_error(e.what());
        return -2;
    }
    double2* base = nullptr;
    rc = noalloc_scratch(&base);
    if (rc) return rc;
    configure_once();
    cudaStream_t st = (cudaStream_t)stream;
    double2 tw[3 * kNoAllocMaxEdge];
    host_twiddles(n1, tw);
    host_twiddles(n2, tw + n1);
    host_twiddles(n3, tw + n1 + n2);
    double cs[162];
    for (int i = 0; i < 81; i++) { cs[i] = c0[i]; cs[81 + i] = s0[i]; }
    double2* dtw = base + kNoAllocTw;
    double* dcs = reinterpret_cast<double*>(base + kNoAllocCs);
    int* derr = reinterpret_cast<int*>(base + kNoAllocErr);
    // the spectrum is fully written by the first pass; only the error word must start at zero
    if (cudaMemcpyAsync(dtw, tw, (size_t)(n1 + n2 + n3) * sizeof(double2), cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(dcs, cs, sizeof(cs), cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemsetAsync(derr, 0, sizeof(int), st) != cudaSuccess) {
        set_last_error("evp_green_apply_noalloc: copy to the scratch failed");
        return -6;
    }
    Dev d{};
    d.n1 = n1; d.n2 = n2; d.n3 = n3;
    d.n1h = n1 / 2 + 1;
    d.N = (long long)n1 * n2 * n3;
    d.spec = base;
    d.tw1 = dtw; d.tw2 = dtw + n1; d.tw3 = dtw + n1 + n2;
    d.err = derr;
    launch_green_apply(d, pl1, pl2, pl3, d_tau, d_out, dcs, dcs + 81, st);
    int herr = 0;
    cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaError_t ce = cudaStreamSynchronize(st);
    if (ce != cudaSuccess) {
        set_last_error(std::string("evp_green_apply_noalloc: ") + cudaGetErrorString(ce));
        return -6;
    }
    if (herr) {
        set_last_error("evp_green_apply_noalloc: singular acoustic tensor");
        return -3;
    }
    return 0;
}
