// evp_solver.cu -- host orchestration of one LS-EVPFFT solve on a B200 and the C ABI.
//
// The macrostep / equilibrium-iteration control flow of lsevpfft/src/LS-EVPFFT.f90
// runs here on the host; every per-voxel and per-frequency loop runs on the
// device (evp_kernels.cu, evp_fft.cu).  Per equilibrium iteration the host
// launches seven kernels and reads back one small block of sums; the serial
// 6x6 / 3x3 tails of the reference (state_6x6_evpsc, calc_velgradavg_corr,
// calc_c0, convergence and time-step control) run on those sums in FP64.
#include "../../include/evp.h"
#include "evp_deck.h"
#include "evp_batch.h"
#include "evp_dev.cuh"
#include "evp_engine.h"
#include "evp_math.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <filesystem>
#include <functional>
#include <future>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <string>
#include <thread>
#include <vector>
#include <sys/stat.h>

namespace evp {

static thread_local std::string g_last_error;
void set_last_error(const std::string& m) { g_last_error = m; }


#define CK(x)                                                                                              \
    do {                                                                                                   \
        cudaError_t e_ = (x);                                                                              \
        if (e_ != cudaSuccess) throw SolveError(std::string("CUDA error: ") + cudaGetErrorString(e_), -6); \
    } while (0)

void mkdir_p(const std::string& dir) {
    std::string cur;
    for (size_t i = 0; i <= dir.size(); i++) {
        if (i == dir.size() || dir[i] == '/')
            if (!cur.empty()) ::mkdir(cur.c_str(), 0755);
        if (i < dir.size()) cur += dir[i];
    }
}
static std::string g0(double x) {
    char b[40];
    std::snprintf(b, sizeof(b), "%.17g", x);
    return b;
}
// Fortran E18.8E3 (write_vtk_cell)
static void put_e18(std::string& o, double x) {
    if (std::fabs(x) < EVP_TINY) x = 0.0;  // clamp_subnormal (IO_functions.f90:938-943)
    char m[40], b[40];
    if (x == 0.0) {
        std::snprintf(b, sizeof(b), "%18s", "0.00000000E+000");
        o += b;
        return;
    }
    std::snprintf(m, sizeof(m), "%.7e", std::fabs(x));
    int e10 = std::atoi(m + 10) + 1;
    char dg[9];
    dg[0] = m[0];
    std::memcpy(dg + 1, m + 2, 7);
    dg[8] = 0;
    char body[40];
    std::snprintf(body, sizeof(body), "%s0.%sE%c%03d", x < 0 ? "-" : "", dg, e10 < 0 ? '-' : '+', e10 < 0 ? -e10 : e10);
    std::snprintf(b, sizeof(b), "%18s", body);
    o += b;
}

struct Diag {
    double detF_min = 0, detF_min_sol = 0, detF_min_gas = 0, detF_min_prev = 0, detF_min_sol_prev = 0, detF_min_gas_prev = 0;
    double detF_min_sol_rel = 0, detF_min_gas_rel = 0;
    double volinc_sol = 0, volinc_gas = 0, volinc_sol_prev = 0, volinc_gas_prev = 0, volinc_sol_rel = 0, volinc_gas_rel = 0;
    double stretch_sol = 0, stretch_gas = 0, stretch_sol_prev = 0, stretch_gas_prev = 0, stretch_sol_rel = 0, stretch_gas_rel = 0;
    double rot_sol = 0, rot_gas = 0;
    double dl_rms_sol = 0, dl_rms_gas = 0, dl_rms = 0, dl_max_sol = 0, dl_max_gas = 0, dl_max = 0;
    double dvelgradavg_mag = 0, erre = 0, errs = 0, errsbc = 0, tdotref = 0, devm_inc_max = 0, s33_target = 0, s33 = 0, s33_sol = 0;
    double cond_sol = 0, cond_gas = 0, cond_cgas = 0;
    int imin_sol[3] = {0, 0, 0}, imin_gas[3] = {0, 0, 0};
};
// Iterations in one round: the expected count rounded down to a power of two and capped, so
// that an engine holds at most four captured graphs (1, 2, 4 and 8 iterations).
static constexpr int kMaxRound = 8;
static int round_length(int want) {
    int k = 1;
    while (2 * k <= want && k < kMaxRound) k *= 2;
    return k;
}

static double safe_rel(double x, double xp) { return (xp <= EVP_TINY || xp >= EVP_HUGE * 0.5) ? 0.0 : std::fabs(x - xp) / xp; }

class Solver {
public:
    Deck dk;
    Dev d{};
    cudaStream_t st = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    FftPlan1D pl1{}, pl2{}, pl3{};
    std::vector<void*> allocs;
    double* h_red = nullptr;  // pinned copy of the result buffer
    int* h_err = nullptr;
    IterCtl* d_ctl = nullptr;  // control block of the equilibrium iteration (device) and its pinned host copy
    IterCtl* h_ctl = nullptr;
    bool own_stream = true;
    bool did_converge = false, accept_step = false;
    double *d_c0 = nullptr, *d_s0 = nullptr, *d_g0 = nullptr;
    // macro state (micro_type, types.f90:55-94)
    double c066[36] = {}, s066[36] = {}, c0[81] = {}, s0[81] = {}, de_ds[81] = {}, goperr0[81] = {};
    double wphsol = 0, wphgas = 0, wphcsol = 0, wphcgas = 0;
    double defgradavg[9], dinvc[9], dinvcs[9], dinvcg[9];
    double dvelgradavg[9] = {}, velgradavg[9] = {}, velgradavgsol[9] = {}, velgradavggas[9] = {};
    double sgavg[9] = {}, sgavgsol[9] = {}, sgsolavg[9] = {};
    double svmavg = 0, dvmavg = 0, edotvmmx = 0, evmavg = 0, evmpavg = 0, dvmpavg = 0, lvmavg = 0;
    double epavg[9] = {}, eavg[9] = {}, eelavg[9] = {}, edotpavg[9] = {};
    Diag dg;
    // driver state (global.f90:19-27, LS-EVPFFT.f90:15-82)
    int ipr = 0, imacroloop = 1, imicro = 0, iter = 0, nconverged = 0, total_macrosteps = 0;
    double erre = 0, errs = 0, errsbc = 0, mix = 1.0, sim_time = 0, wall_time = 0, tdot_plan = 0, proc_time_target = 0,
           proc_time_done = 0;
    bool kinematic = false, do_mix = true, modal = false, write_files = false, verbose = false, finished = false;
    long long vlast = -1;
    long long total_iters = 0;
    int macrosteps_done = 0;
    double gpu_ms = 0.0;
    std::time_t start = 0;
    std::string outdir;
    double last_results[51] = {}, last_diag[44] = {};
    std::vector<double> snap_dsim, snap_scau;
    bool has_thermo = false;
    std::vector<double> eth_soa;  // host staging of the thermal eigenstrain upload (kept until the copy completes)
    // optional wall-clock budget: the solve ends with -8 at the first equilibrium iteration after it
    bool has_deadline = false;
    std::chrono::steady_clock::time_point deadline{};
    void check_deadline() const {
        if (has_deadline && std::chrono::steady_clock::now() > deadline)
            throw SolveError("deadline exceeded: the solve's wall-clock budget ran out", -8);
    }

    ProcessData& P() { return dk.process[ipr - 1]; }

    template <class T>
    T* dalloc(size_t n) {
        void* p = nullptr;
        if (n == 0) return nullptr;
        // stream-ordered from the library's own pool: no device-wide sync, so concurrent solves do not stall
        CK(cudaMallocFromPoolAsync(&p, n * sizeof(T), evp::solver_pool(), st));
        allocs.push_back(p);
        return (T*)p;
    }
    ~Solver() {
        if (vtk_job.valid()) {
            try {
                vtk_job.get();
            } catch (...) {
            }
        }
        solo.reset();
        for (void* p : allocs) cudaFreeAsync(p, st);
        if (st) cudaStreamSynchronize(st);
        if (h_red) cudaFreeHost(h_red);
        if (h_err) cudaFreeHost(h_err);
        if (h_ctl) cudaFreeHost(h_ctl);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (st && own_stream) cudaStreamDestroy(st);
        for (auto& p : pend) {
            cudaEventDestroy(p.a);
            cudaEventDestroy(p.b);
        }
        for (auto e : evpool) cudaEventDestroy(e);
    }

    // ---- host<->device byte counters and the optional per-kernel event timer
    long long h2d = 0, d2h = 0;
    bool profile = false, write_vtk_files = false;
    // VTK files are formatted and written by a background task (one at a time) while the solve
    // goes on, when the caller only needs the files at the end of the solve (evp_solve_file, a
    // batch or server member); wait_vtk() finishes the last one and reports its error.
    bool async_vtk = false;
    std::future<void> vtk_job;
    void wait_vtk() {
        if (vtk_job.valid()) vtk_job.get();
    }
    int prec = 0;  // 1: mixed precision (FP32 spectrum, FFTs and Green operator in the equilibrium chain)
    // Mixed precision falls back to FP64 for the rest of an increment once its FP32 iterations stop
    // reducing the error: the FP32 round-off of the Green-operator update is about 1e-7 of the stress
    // heterogeneity, which can exceed the tolerance when the strain rates are very small (slow creep).
    int prec_it = 0;
    // Mixed precision: an increment whose FP32 iterations stagnated (it finished in FP64) makes
    // the next increments start in FP64; FP32 is tried again after 2, 4, ... 32 increments.
    bool inc_fp32 = false;  // this increment started with FP32 spectra
    int fp64_hold = 0;      // increments still to start in FP64
    int fp64_len = 2;       // length of the next hold
    std::vector<double> err_hist;
    struct KTime {
        std::string name;
        long long n = 0;
        double ms = 0.0;
    };
    std::vector<KTime> ktimes;
    struct Pending {
        int k;
        cudaEvent_t a, b;
    };
    std::vector<Pending> pend;
    std::vector<cudaEvent_t> evpool;
    cudaEvent_t get_ev() {
        if (!evpool.empty()) { cudaEvent_t e = evpool.back(); evpool.pop_back(); return e; }
        cudaEvent_t e;
        CK(cudaEventCreate(&e));
        return e;
    }
    long long launches = 0;  // kernels launched by this solve (K() wrappers; k_grid_fft counts its five passes)
    template <class F>
    void K(const char* name, F&& f, int nlaunch = 1) {
        launches += nlaunch;
        if (!profile) { f(); return; }
        int k = -1;
        for (size_t i = 0; i < ktimes.size(); i++)
            if (ktimes[i].name == name) { k = (int)i; break; }
        if (k < 0) { ktimes.push_back(KTime{name}); k = (int)ktimes.size() - 1; }
        cudaEvent_t a = get_ev(), b = get_ev();
        CK(cudaEventRecord(a, st));
        f();
        CK(cudaEventRecord(b, st));
        pend.push_back(Pending{k, a, b});
    }
    void resolve_timers() {
        for (auto& p : pend) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) { ktimes[p.k].n++; ktimes[p.k].ms += ms; }
            evpool.push_back(p.a);
            evpool.push_back(p.b);
        }
        pend.clear();
    }
    void h2d_copy(void* dst, const void* src, size_t bytes) {
        CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
        h2d += (long long)bytes;
    }

    void sync() { CK(cudaStreamSynchronize(st)); }
    // the result buffer and the error word to the host: queued (fetch_red_async), then read after
    // the stream is synchronised (check_red); fetch_red does both
    void fetch_red_async() {
        CK(cudaMemcpyAsync(h_red, d.red, RED_OUT_SIZE * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(h_err, d.err, sizeof(int), cudaMemcpyDeviceToHost, st));
        d2h += RED_OUT_SIZE * sizeof(double) + sizeof(int);
    }
    void check_red() {
        resolve_timers();
        if (*h_err & 1) throw SolveError("singular matrix in a voxel operator (lu_inverse / lu_eqsystem)", -3);
        if (*h_err & 2) throw SolveError("non-finite stress in the local Newton solve", -4);
        if (*h_err & 4) throw SolveError("form_G failed (singular acoustic tensor or complex D operator)", -3);
        if (*h_err & 8) throw SolveError("a bulk copy into shared memory did not complete", -6);
    }
    void fetch_red() {
        fetch_red_async();
        sync();
        check_red();
    }

    // Device memory comes stream-ordered from the library's own pool (solver_pool): no
    // device-wide synchronisation, so solves running beside each other do not stall, and
    // back-to-back solves reuse the memory.

    // ------------------------------------------------------------ open (LS-EVPFFT.f90:144-178)
    // ext_stream: run on the caller's stream (a batch's); parsed: the deck, already read (the
    // server parses decks on the submitting thread)
    void open(const std::string& fft_in, const std::string& out, int mix_flag, int modal_flag, int flags,
              cudaStream_t ext_stream = nullptr, Deck* parsed = nullptr) {
        write_files = (flags & (EVP_WRITE_FILES | EVP_WRITE_CSV)) != 0;
        write_vtk_files = (flags & EVP_WRITE_FILES) != 0;
        profile = (flags & EVP_PROFILE) != 0;
        prec = (flags & EVP_MIXED) ? 1 : 0;
        verbose = (flags & EVP_VERBOSE) != 0;
        outdir = out.empty() ? std::string("evpfft_outputs/") : out;
        if (write_files) {
            mkdir_p(outdir);
            // old *.vtk / *.out are removed at start (LS-EVPFFT.f90:145-146): regular files directly
            // in the output directory, no shell involved
            std::error_code ec;
            for (const auto& e : std::filesystem::directory_iterator(outdir, ec)) {
                const std::string ext = e.path().extension().string();
                std::error_code ec2;
                if ((ext == ".vtk" || ext == ".out") && e.is_regular_file(ec2)) std::filesystem::remove(e.path(), ec2);
            }
        }
        if (parsed) {
            dk = std::move(*parsed);
        } else {
            try {
                dk = parse_deck(fft_in);
            } catch (DeckError& e) {
                throw SolveError(e.what(), e.code);
            }
        }
        int dev_count = 0;
        if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0) throw SolveError("no CUDA device available", -6);
        if (ext_stream) {
            st = ext_stream;
            own_stream = false;
        } else {
            CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        }
        CK(cudaEventCreate(&ev0));
        CK(cudaEventCreate(&ev1));
        static std::once_flag configured;
        std::call_once(configured, [] { fft_configure(); });
        allocate();
        upload_and_init();
        modal = (modal_flag != 0);
        do_mix = (mix_flag != 0);
        start = std::time(nullptr);
        const ProcessData& p1 = dk.process[0];
        dvmavg = vm_strain(p1.dsim);
        lvmavg = dvmavg;
        if (write_vtk_files) write_vtk(0);
        // start-up tangent (LS-EVPFFT.f90:156-173)
        for (int c = 0; c < 36; c++) c066[c] = h_red[OFF_INIT + c] / wphcsol * p1.tdot;
        for (int c = 0; c < 36; c++) s066[c] = c066[c];
        if (lu_inverse(s066, 6) != 0) throw SolveError("Singular matrix in lu_inverse (start-up c066)", -3);
        b66_to_t4(c066, c0);
        b66_to_t4(s066, s0);
        std::memcpy(de_ds, s0, sizeof(de_ds));
        upload_c0();
        fft_autotune(d, pl1, pl2, pl3, d_c0, d_s0, prec, st);  // once per grid and process
        if (write_files) write_headers();
        for (auto& p : dk.process) total_macrosteps += p.nsteps;
        imacroloop = 1;
        ipr = 0;
        imicro = 0;
    }

    void allocate() {
        const long long N = dk.nvox();
        d.N = N;
        d.n1 = dk.n1; d.n2 = dk.n2; d.n3 = dk.n3;
        d.n1h = dk.n1 / 2 + 1;
        d.n3node = (dk.n3 == 1) ? 1 : dk.n3 + 1;
        d.wgt = dk.wgt;
        int ns = 1;
        for (auto& ph : dk.phase) ns = std::max(ns, ph.nsyst);
        d.nsys = ns;
        long long g = (N + 255) / 256;
        d.grid = (int)std::min<long long>(g, 148LL * 8);
        d.sg = dalloc<double>(6 * N); d.sgt = dalloc<double>(6 * N); d.edotp = dalloc<double>(6 * N);
        d.ept = dalloc<double>(6 * N); d.disgradsym = dalloc<double>(6 * N);
        d.velgrad = dalloc<double>(9 * N); d.velgradold = dalloc<double>(9 * N); d.dvr = dalloc<double>(9 * N);
        d.F = dalloc<double>(9 * N); d.Finv = dalloc<double>(9 * N); d.Fe = dalloc<double>(9 * N); d.Fp = dalloc<double>(9 * N);
        d.Finc = dalloc<double>(9 * N); d.Feinc = dalloc<double>(9 * N); d.ag = dalloc<double>(9 * N);
        d.detF = dalloc<double>(N); d.wgtc = dalloc<double>(N); d.epvm = dalloc<double>(N); d.gacumgr = dalloc<double>(N);
        d.sg66 = dalloc<double>(36 * N); d.c066mod = dalloc<double>(36 * N); d.c066inv = dalloc<double>(36 * N);
        d.cG = dalloc<double>(36 * N);
        d.cgas = dk.has_gas ? dalloc<double>(36 * N) : nullptr;
        d.sch = dalloc<double>(5 * (size_t)ns * N);
        d.crss = dalloc<double>(2 * (size_t)ns * N); d.trialtau = dalloc<double>(2 * (size_t)ns * N);
        d.gamdot = dalloc<double>((size_t)ns * N);
        d.eth = dk.eth.empty() ? nullptr : dalloc<double>(9 * N);
        d.gas = dalloc<uint8_t>(N); d.phase = dalloc<uint8_t>(N);
        d.s_velgrad = dalloc<double>(9 * N); d.s_velgradold = dalloc<double>(9 * N); d.s_sg = dalloc<double>(6 * N);
        d.s_edotp = dalloc<double>(6 * N); d.s_gamdot = dalloc<double>((size_t)ns * N); d.s_trialtau = dalloc<double>(2 * (size_t)ns * N);
        d.spec = dalloc<double2>(9 * (size_t)d.n1h * dk.n2 * dk.n3);
        {
            bool any_tab = false;
            for (auto& p : dk.process) any_tab = any_tab || p.igamma != 0;
            d.goper = any_tab ? dalloc<double>(81 * (size_t)d.n1h * dk.n2 * dk.n3) : nullptr;
            d.gtab = 0;
        }
        d.tw1 = dalloc<double2>(dk.n1); d.tw2 = dalloc<double2>(dk.n2); d.tw3 = dalloc<double2>(dk.n3);
        d.dv3 = dalloc<double>(3 * N);
        d.Fini = dk.idispini > 0 ? dalloc<double>(9 * N) : nullptr;
        d.xnode = dalloc<double>(3 * (size_t)(dk.n1 + 1) * (dk.n2 + 1) * d.n3node);
        // block partials: voxel kernels (<= 1184 blocks x 117 sums), Newton (<= 3552 x 14), and the
        // x inverse pass (one block per <= 1 pair of rows x 9 sums)
        d.partials = dalloc<double>(std::max<size_t>(200 * 2048, 9 * ((size_t)dk.n2 * dk.n3 / 2 + 1)));
        d.red = dalloc<double>(RED_OUT_SIZE);
        d.counters = dalloc<unsigned int>(CNT_N);
        d.err = dalloc<int>(1);
        d.nstats = profile ? dalloc<unsigned long long>(8) : nullptr;
        if (d.nstats) CK(cudaMemsetAsync(d.nstats, 0, 8 * sizeof(unsigned long long), st));
        CK(cudaMemsetAsync(d.counters, 0, CNT_N * sizeof(unsigned int), st));
        CK(cudaMemsetAsync(d.err, 0, sizeof(int), st));
        CK(cudaMemsetAsync(d.red, 0, RED_OUT_SIZE * sizeof(double), st));
        CK(cudaMemsetAsync(d.cG, 0, 36 * N * sizeof(double), st));
        d_c0 = dalloc<double>(81); d_s0 = dalloc<double>(81); d_g0 = dalloc<double>(81);
        CK(cudaMemsetAsync(d_g0, 0, 81 * sizeof(double), st));
        CK(cudaMallocHost(&h_red, RED_OUT_SIZE * sizeof(double)));
        CK(cudaMallocHost(&h_err, sizeof(int)));
        CK(cudaMallocHost(&h_ctl, sizeof(IterCtl)));
        std::memset(h_ctl, 0, sizeof(IterCtl));
        d_ctl = dalloc<IterCtl>(1);
        CK(cudaMemsetAsync(d_ctl, 0, sizeof(IterCtl), st));
        pl1 = make_plan(dk.n1); pl2 = make_plan(dk.n2); pl3 = make_plan(dk.n3);
        auto twiddles = [&](int n, double2* dst) {
            std::vector<double2> t(n);
            for (int e = 0; e < n; e++) {
                long double ang = -2.0L * 3.14159265358979323846264338327950288L * (long double)e / (long double)n;
                t[e] = make_double2((double)cosl(ang), (double)sinl(ang));
            }
            h2d_copy(dst, t.data(), n * sizeof(double2));
            sync();
        };
        twiddles(dk.n1, d.tw1); twiddles(dk.n2, d.tw2); twiddles(dk.n3, d.tw3);
        if (prec) {  // FP32 copies, rounded from the same long-double angles
            auto twiddles_f = [&](int n, float2* dst) {
                std::vector<float2> t(n);
                for (int e = 0; e < n; e++) {
                    long double ang = -2.0L * 3.14159265358979323846264338327950288L * (long double)e / (long double)n;
                    t[e] = make_float2((float)cosl(ang), (float)sinl(ang));
                }
                h2d_copy(dst, t.data(), n * sizeof(float2));
            };
            d.tw1f = dalloc<float2>(dk.n1); d.tw2f = dalloc<float2>(dk.n2); d.tw3f = dalloc<float2>(dk.n3);
            twiddles_f(dk.n1, d.tw1f); twiddles_f(dk.n2, d.tw2f); twiddles_f(dk.n3, d.tw3f);
        }
        // phases
        std::vector<PhaseDev> ph(dk.nph);
        for (int p = 0; p < dk.nph; p++) {
            const PhaseData& s = dk.phase[p];
            PhaseDev& t = ph[p];
            std::memset(&t, 0, sizeof(t));
            t.nsyst = s.nsyst; t.nmodes = s.nmodes; t.igas = s.igas ? 1 : 0;
            t.int_exp = 1;
            for (int m = 0; m < 3; m++) t.nsm[m] = s.nsm[m];
            int islast = 0;
            for (int m = 0; m < s.nmodes; m++) {
                islast += s.nsm[m];
                t.tau1[m] = s.tau[islast - 1][2];
                t.thet0[m] = s.thet[islast - 1][0];
                t.thet1[m] = s.thet[islast - 1][1];
            }
            for (int i = 0; i < kMaxSys; i++) {
                t.nrs[i] = s.nrs[i]; t.gamd0[i] = s.gamd0[i]; t.hpfac[i] = s.hpfac[i];
                t.tau0f[i] = s.tau[i][0]; t.tau0b[i] = s.tau[i][1];
                for (int j = 0; j < kMaxSys; j++) t.hard[i * kMaxSysDev + j] = s.hard[i][j];
                for (int c = 0; c < 3; c++) { t.dnca[3 * i + c] = s.dnca[i][c]; t.dbca[3 * i + c] = s.dbca[i][c]; }
                if (i < s.nsyst) {
                    double e = s.nrs[i] - 1.0;
                    if (!(e >= 0.0 && e <= 64.0 && e == std::floor(e))) t.int_exp = 0;
                }
            }
            for (int c = 0; c < 81; c++) t.C[c] = s.C[c];
        }
        PhaseDev* dph = dalloc<PhaseDev>(dk.nph);
        h2d_copy(dph, ph.data(), dk.nph * sizeof(PhaseDev));
        d.ph = dph;
        d.nph = dk.nph;
    }

    // init_defgrad (IO_functions.f90:815-936): F = grad(u) + diag(delt) (delt forced to 4), the
    // spectral gradient with ideriv = IDISPINI; the macroscopic weights and inverse averages.
    // velgradold and dvr are scratch here (k_init clears both afterwards).
    void init_defgrad(double& detFavg) {
        const long long N = d.N;
        std::vector<double> u9(9 * (size_t)N);
        for (int m = 0; m < 3; m++)
            for (int l = 0; l < 3; l++)
                for (long long v = 0; v < N; v++) u9[(size_t)(3 * m + l) * N + v] = dk.dispini[3 * (size_t)v + l];
        h2d_copy(d.velgradold, u9.data(), u9.size() * sizeof(double));
        K("k_gradient", [&] { launch_gradient(d, pl1, pl2, pl3, d.velgradold, d.dvr, dk.idispini, st); });
        K("k_dispini", [&] { launch_dispini(d, d.dvr, 4.0, st); });
        fetch_red();
        const double* S = h_red + OFF_DISP;
        detFavg = S[29];
        wphcsol = S[27] / detFavg;
        wphcgas = S[28] / detFavg;
        for (int c = 0; c < 9; c++) {
            const double id = (c % 4 == 0) ? 1.0 : 0.0;
            defgradavg[c] = 4.0 * id;  // diag(delt)
            dinvc[c] = S[c] / detFavg;
            dinvcs[c] = S[9 + c] / detFavg / wphcsol;
            dinvcg[c] = (wphcgas > 0.0) ? S[18 + c] / detFavg / wphcgas : id;
        }
    }

    void upload_and_init() {
        const long long N = d.N;
        std::vector<uint8_t> gas(N), phs(N);
        wphsol = 0.0; wphgas = 0.0;
        for (long long v = 0; v < N; v++) {
            phs[v] = (uint8_t)(dk.phase_id[v] - 1);
            gas[v] = dk.phase[dk.phase_id[v] - 1].igas ? 1 : 0;
            if (gas[v]) wphgas += dk.wgt;
            if (!gas[v]) { wphsol += dk.wgt; vlast = v; }
        }
        wphcsol = wphsol;
        wphcgas = wphgas;
        for (int c = 0; c < 9; c++) {
            defgradavg[c] = dinvc[c] = dinvcs[c] = dinvcg[c] = (c % 4 == 0) ? 1.0 : 0.0;
        }
        h2d_copy(d.gas, gas.data(), N);
        h2d_copy(d.phase, phs.data(), N);
        if (d.eth) {  // the deck keeps eth voxel-major (9 per voxel); the device field is component-major
            eth_soa.resize(9 * (size_t)N);
            for (long long v = 0; v < N; v++)
                for (int c = 0; c < 9; c++) eth_soa[(size_t)c * N + v] = dk.eth[9 * (size_t)v + c];
            h2d_copy(d.eth, eth_soa.data(), 9 * N * sizeof(double));
        }
        for (auto& p : dk.process) has_thermo = has_thermo || p.ithermo == 1;
        double* d_eul = dalloc<double>(3 * N);
        int* d_gr = dalloc<int>(N);
        double* d_hp = dalloc<double>(N);
        h2d_copy(d_eul, dk.euler.data(), 3 * N * sizeof(double));
        h2d_copy(d_gr, dk.grain.data(), N * sizeof(int));
        h2d_copy(d_hp, dk.hp_shift.data(), N * sizeof(double));
        // xnode start values (types.f90:273-287)
        {
            const int n1 = dk.n1, n2 = dk.n2, nn3 = d.n3node;
            std::vector<double> xn(3 * (size_t)(n1 + 1) * (n2 + 1) * nn3);
            for (int k = 0; k < nn3; k++)
                for (int j = 0; j < n2 + 1; j++)
                    for (int i = 0; i < n1 + 1; i++) {
                        size_t p = 3 * (i + (size_t)(n1 + 1) * (j + (size_t)(n2 + 1) * k));
                        xn[p] = (double)(i + 1) - 0.5;
                        xn[p + 1] = (double)(j + 1) - 0.5;
                        xn[p + 2] = (nn3 == 1) ? 0.0 : (double)(k + 1) - 0.5;
                    }
            if (dk.idispini > 0)  // xnode + dispini_node (IO_functions.f90:885); same node layout
                for (size_t q = 0; q < xn.size(); q++) xn[q] = xn[q] + dk.dispini_node[q];
            h2d_copy(d.xnode, xn.data(), xn.size() * sizeof(double));
        }
        double detFavg = 1.0;
        if (dk.idispini > 0) init_defgrad(detFavg);
        const ProcessData& p1 = dk.process[0];
        double u6[6], u6t[6];
        t2_to_b6(p1.udot, u6);
        for (int c = 0; c < 6; c++) u6t[c] = u6[c] * p1.tdot;
        launch_init(d, d_eul, d_gr, d_hp, p1.udot, u6t, dk.idispini > 0 ? 1 : 0, detFavg, st);
        CK(cudaGetLastError());
        fetch_red();
        // release the start-up staging buffers
        for (void* p : {(void*)d_eul, (void*)d_gr, (void*)d_hp}) {
            CK(cudaFreeAsync(p, st));
            allocs.erase(std::find(allocs.begin(), allocs.end(), p));
        }
    }

    void upload_c0() {
        h2d_copy(d_c0, c0, sizeof(c0));
        h2d_copy(d_s0, s0, sizeof(s0));
    }

    // ------------------------------------------------------------ snapshots (various_functions.f90:2839-2895)
    void snapshot(bool take) {
        const long long N = d.N;
        const size_t ns = d.nsys;
        auto cp = [&](double* dst, double* src, size_t n) {
            CK(cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
        };
        ProcessData& p = P();
        if (take) {
            snap_dsim.assign(p.dsim, p.dsim + 9);
            snap_scau.assign(p.scauchy, p.scauchy + 9);
            cp(d.s_velgrad, d.velgrad, 9 * N); cp(d.s_velgradold, d.velgradold, 9 * N); cp(d.s_sg, d.sg, 6 * N);
            cp(d.s_edotp, d.edotp, 6 * N); cp(d.s_gamdot, d.gamdot, ns * N); cp(d.s_trialtau, d.trialtau, 2 * ns * N);
        } else {
            std::memcpy(p.dsim, snap_dsim.data(), 9 * sizeof(double));
            std::memcpy(p.scauchy, snap_scau.data(), 9 * sizeof(double));
            cp(d.velgrad, d.s_velgrad, 9 * N); cp(d.velgradold, d.s_velgradold, 9 * N); cp(d.sg, d.s_sg, 6 * N);
            cp(d.edotp, d.s_edotp, 6 * N); cp(d.gamdot, d.s_gamdot, ns * N); cp(d.trialtau, d.s_trialtau, 2 * ns * N);
        }
    }

    // ------------------------------------------------------------ the increment's iteration control block
    // Fill the control block for the first iteration of an increment (the iter == 0 block of
    // LS-EVPFFT.f90:233-240, and what equilibrium_iteration reads from the driver) and upload it.
    void start_iterations() {
        ProcessData& p = P();
        if (dk.has_gas) K("k_gas_compl", [&] { launch_gas_compl(d, p.tdot, dk.complgas, modal ? 1 : 0, st); });
        std::memset(dvelgradavg, 0, sizeof(dvelgradavg));
        edotvmmx = 0;
        mix = 1.0;
        erre = 2.0 * p.error;
        errs = 2.0 * p.error;
        errsbc = 2.0 * p.error;
        inc_fp32 = prec != 0 && fp64_hold == 0;
        prec_it = inc_fp32 ? 1 : 0;
        IterCtl& c = *h_ctl;
        std::memset(&c, 0, sizeof(c));
        c.active = 1;
        c.prec = prec_it;
        c.fresh = 1;
        c.sg_off = OFF_SGAVG;
        c.corr.mix = mix;
        c.corr.Lscale = std::max(lvmavg, EVP_TINY);
        c.corr.do_mix = do_mix ? 1 : 0;
        c.corr.kinematic = kinematic ? 1 : 0;
        if (inv3(dinvc, c.xinv.dinv) != 0) throw SolveError("Singular matrix in lu_inverse (correction_to_current)", -3);
        c.newton.tdot = p.tdot;
        c.newton.error = p.error;
        c.newton.erroral = p.erroral;
        c.newton.complgas = dk.complgas;
        c.newton.modal = modal ? 1 : 0;
        c.newton.thermo = (imicro == 1 && p.ithermo == 1) ? 1 : 0;
        c.newton.iuphard = p.iuphard;
        c.iter = 0;
        c.itmax = p.itmax;
        c.ictrl = p.ictrl;
        c.kinematic = kinematic ? 1 : 0;
        c.total_iters = total_iters;
        c.error = p.error;
        c.tdotmin = p.tdotmin;
        c.devmapp = p.devmapp;
        c.lvmavg = lvmavg;
        c.erre = erre;
        c.errs = errs;
        c.errsbc = errsbc;
        c.svmavg = svmavg;
        c.wphcsol = wphcsol;
        c.wphcgas = wphcgas;
        std::memcpy(c.velgradavg, velgradavg, sizeof(velgradavg));
        // the increment's constants of state_6x6_evpsc (various_functions.f90:1638-1705): de_ds in the
        // b-basis, its Voigt form and the LU factors of the mixed-BC system, formed by the same
        // functions the per-iteration tail used to call, so every bit is as before
        {
            double a4[81];
            t4_to_b66(de_ds, c.mev);
            b66_to_t4(c.mev, a4);
            for (int i = 0; i < 6; i++)
                for (int j = 0; j < 6; j++) c.xmv[6 * i + j] = a4[(3 * ijv_a(i) + ijv_b(i)) * 9 + 3 * ijv_a(j) + ijv_b(j)];
            double profac[6];
            for (int i = 1; i <= 6; i++) profac[i - 1] = 1.0 + (i / 4);
            for (int i = 0; i < 6; i++)
                for (int j = 0; j < 6; j++)
                    c.lu[6 * i + j] = p.iscau[j] * (i == j ? 1 : 0) - p.idsim[j] * c.xmv[6 * i + j] * profac[j];
            if (lu_factor(c.lu, 6, c.piv) != 0) throw SolveError("Failed system solve in lu_eqsystem (state_6x6_evpsc)", -3);
        }
        for (int i = 0; i < 6; i++) {
            c.iscau[i] = p.iscau[i];
            c.idsim[i] = p.idsim[i];
        }
        for (int k = 0; k < 9; k++) {
            c.iudot[k] = p.iudot[k];
            c.udot[k] = p.udot[k];
            c.dsim[k] = p.dsim[k];
            c.scauchy[k] = p.scauchy[k];
        }
        c.tdot = p.tdot;
        c.tdotref = p.tdotref;
        h2d_copy(d_ctl, h_ctl, sizeof(IterCtl));
        // the weighted stress average the first iteration starts from (LS-EVPFFT.f90:238-252; later
        // iterations take it from the previous Newton launch's sums of the same stresses)
        K("k_sgavg", [&] { launch_sgavg(d, st); });
    }

    // The control block back on the host once the device has stopped the iteration (an event).
    void pull_ctl() {
        CK(cudaMemcpyAsync(h_ctl, d_ctl, sizeof(IterCtl), cudaMemcpyDeviceToHost, st));
        d2h += (long long)sizeof(IterCtl);
        sync();
        resolve_timers();
        const IterCtl& c = *h_ctl;
        ProcessData& p = P();
        iter = c.iter;
        total_iters = c.total_iters;
        erre = c.erre;
        errs = c.errs;
        errsbc = c.errsbc;
        svmavg = c.svmavg;
        mix = c.corr.mix;
        prec_it = c.prec;
        std::memcpy(velgradavg, c.velgradavg, sizeof(velgradavg));
        std::memcpy(velgradavggas, c.velgradavggas, sizeof(velgradavggas));
        std::memcpy(velgradavgsol, c.velgradavgsol, sizeof(velgradavgsol));
        std::memcpy(sgavg, c.sgavg, sizeof(sgavg));
        std::memcpy(sgavgsol, c.sgavgsol, sizeof(sgavgsol));
        std::memcpy(dvelgradavg, c.xinv.dvelgradavg, sizeof(dvelgradavg));
        std::memcpy(p.dsim, c.dsim, sizeof(c.dsim));
        std::memcpy(p.scauchy, c.scauchy, sizeof(c.scauchy));
        p.tdot = c.tdot;
        p.tdotref = c.tdotref;
        if (verbose) {
            std::printf("\rMACROSTEP=%d SimTime=%.0fs PROC=%d STEP=%d TDOT=%.0fs ITER=%d", imacroloop, sim_time, ipr, imicro,
                        p.tdot, iter);
            std::fflush(stdout);
        }
    }

    // Resume the iteration after the host looked at it and changed nothing on the device.
    void resume_iterations() {
        h_ctl->active = 1;
        h_ctl->event = EV_RUNNING;
        h2d_copy(d_ctl, h_ctl, sizeof(IterCtl));
    }

    static std::string ctl_message(int bits) {
        if (bits & 1) return "singular matrix in a voxel operator (lu_inverse / lu_eqsystem)";
        if (bits & 2) return "non-finite stress in the local Newton solve";
        if (bits & 4) return "form_G failed (singular acoustic tensor or complex D operator)";
        if (bits & 8) return "ERRE/ERRS negative -> convergence failed!";
        if (bits & 32) return "equilibrium iteration did not converge";
        if (bits & 64) return "a bulk copy into shared memory did not complete";
        return "equilibrium iteration failed";
    }

    // After an event: true when the increment's iteration loop is over (converged, or accepted
    // at ITMAX), false when it goes on (iterations resumed or restarted from the snapshot).
    // The ictrl = -1 sub-stepping decision of LS-EVPFFT.f90:378-427 runs here.
    bool handle_event(int ev) {
        if (ev < 0) throw SolveError(ctl_message(h_ctl->errbits), ev);
        ProcessData& p = P();
        did_converge = h_ctl->did_converge != 0;
        accept_step = false;
        if (ev == EV_CONVERGED) return true;
        if (ev == EV_ACCEPTED) {
            accept_step = true;
            return true;
        }
        // EV_HOST: ictrl = -1 with tdot above tdotmin, at convergence or at ITMAX
        bool restart = false;
        double md;
        if (!did_converge && iter == p.itmax) {
            double tdot = p.tdot;
            int nsub = kinematic_substep(tdot, md);
            tdot = tdot / nsub;
            tdot = std::max(p.tdotmin, std::min(tdot, 0.5 * p.tdot));
            nsub = (int)std::ceil(p.tdot / tdot);
            if (nsub > 1) {
                const double remaining = std::max(0.0, proc_time_target - proc_time_done);
                tdot_plan = tdot;
                const int nnew = (imicro - 1) + (int)std::ceil(remaining / tdot_plan);
                total_macrosteps += nnew - p.nsteps;
                p.nsteps = nnew;
                p.tdot = std::min(tdot_plan, remaining);
                nconverged = 0;
                restart = true;
            }
        } else if (did_converge) {
            double tdot = p.tdot;
            int nsub = kinematic_substep(tdot, md);
            tdot = tdot / nsub;
            if (md <= 1.0e-3) tdot = std::max(p.tdotmin, std::min(tdot, 0.5 * p.tdot));
            else tdot = std::max(p.tdotmin, tdot);
            nsub = (int)std::ceil(p.tdot / tdot);
            if (nsub > 1) {
                const double remaining = std::max(0.0, proc_time_target - proc_time_done);
                tdot_plan = tdot;
                const int nnew = (imicro - 1) + (int)std::ceil(remaining / tdot_plan);
                total_macrosteps += nnew - p.nsteps;
                p.nsteps = nnew;
                p.tdot = std::min(tdot_plan, remaining);
                did_converge = false;
                nconverged = 0;
                restart = true;
            }
        }
        if (iter >= 100000) throw SolveError("equilibrium iteration did not converge", -4);
        if (restart) {  // roll the increment back and iterate it again with the cut time step
            iter = 0;
            inc_launched = 0;
            snapshot(false);
            start_iterations();
            return false;
        }
        if (did_converge) return true;
        resume_iterations();
        return false;
    }

    int kinematic_substep(double tdot_step, double& min_detF) {
        K("k_kinematic", [&] { launch_kinematic(d, tdot_step, st); });
        CK(cudaGetLastError());
        fetch_red();
        const double mv = h_red[OFF_KIN], mr = h_red[OFF_KIN + 1], ms = h_red[OFF_KIN + 2];
        min_detF = -h_red[OFF_KIN + 3];
        const double worst = std::max(std::max(1.0, mv / 5.0e-2), std::max(mr / 2.0, ms / 5.0e-2));
        return std::max(1, (int)std::ceil(worst));
    }

    // This solve as a member of a batched launch.
    BatchSolve entry() const { return BatchSolve{d, pl1, pl2, pl3, d_ctl, d_c0, d_s0}; }

    // ------------------------------------------------------------ increment start (LS-EVPFFT.f90:199-240)
    // Process switch, time step, snapshot, form_G and the per-increment operators, then the
    // control block of the first iteration.  False once the deck is finished.
    bool begin_increment() {
        while (ipr == 0 || imicro >= P().nsteps) {
            if (ipr >= dk.nproc) { finished = true; return false; }
            ipr++;
            nconverged = 0;
            kinematic = (P().iscau[2] == 0);
            tdot_plan = P().tdot;
            proc_time_target = (double)P().nsteps * tdot_plan;
            proc_time_done = 0.0;
            imicro = 0;
        }
        ProcessData& p = P();
        imicro++;
        CK(cudaEventRecord(ev0, st));
        if (p.ictrl == -1) {
            const double remaining = std::max(0.0, proc_time_target - proc_time_done);
            p.tdot = (remaining > 0.0) ? std::min(tdot_plan, remaining) : tdot_plan;
        }
        snapshot(true);
        did_converge = false;
        accept_step = false;
        const int do_schmid = ((imicro == 1 && ipr == 1) || p.iupdate == 1) ? 1 : 0;
        d.gtab = (p.igamma != 0 && d.goper) ? 1 : 0;
        if (d.gtab) K("k_goper_tab", [&] { launch_goper_tab(d, d_c0, d_s0, p.igamma, st); });  // form_G, IGAMMA 1, 2
        if (modal) {  // form_G: the real-space origin value (IGAMMA 0 is applied on the fly)
            K("k_goperr0", [&] { launch_goperr0(d, d_c0, d_s0, p.igamma, st); });
            fetch_red();
            for (int c = 0; c < 81; c++) goperr0[c] = h_red[OFF_G0 + c] / (double)d.N;
            h2d_copy(d_g0, goperr0, sizeof(goperr0));
        }
        K("k_prologue", [&] { launch_prologue(d, d_c0, d_g0, do_schmid, modal ? 1 : 0, st); });
        iter = 0;
        inc_launched = 0;
        start_iterations();
        return true;
    }

    // ------------------------------------------------------------ increment end (LS-EVPFFT.f90:432-588)
    // end_launch queues the commit, large-strain, diagnostics and calc_c0 kernels and the copy
    // of their sums; end_finish, after the stream has been synchronised, does the host tails
    // and writes the rows.  A batch launches the ends of many solves before one synchronisation.
    struct EndState {
        int iter_done = 0, nsteps_written = 0;
        double tdot_used = 0, tdotref_used = 0;
        bool conv_for_count = false;
    } es;
    void end_launch() {
        ProcessData& p = P();
        es.iter_done = iter;
        prev_inc_iters = iter;
        if (prec) {
            if (!inc_fp32) {
                if (fp64_hold > 0) fp64_hold--;
            } else if (prec_it == 0) {  // fell back to FP64
                fp64_hold = fp64_len;
                fp64_len = std::min(2 * fp64_len, 32);
            } else {
                fp64_len = 2;
            }
        }
        if (p.iupdate == 1) {  // update_grid_velgrad_node reads L and F before update_defgrad changes F
            K("k_grid_fft", [&] {
                launch_fft_x_fwd(d, pl1, 1, 0, st);
                launch_fft_y(d, pl2, 9, false, st);
                launch_fft_z_integ(d, pl3, p.igamma, st);
                launch_fft_y(d, pl2, 3, true, st);
                XinvParams xp{};
                launch_fft_x_inv(d, pl1, 1, xp, st);
            }, 5);
            K("k_cell2node", [&] { launch_cell2node(d, p.tdot, p.igamma, st); });
        }
        Upd1Params u1;
        u1.tdot = p.tdot;
        u1.iupdate = p.iupdate;
        K("k_upd1", [&] { launch_upd1(d, u1, st); });
        if (p.iupdate == 1) {
            Upd2Params u2;
            std::memcpy(u2.velgradavg, velgradavg, sizeof(u2.velgradavg));
            K("k_upd2", [&] { launch_upd2(d, u2, st); });
        }
        Upd3Params u3;
        u3.tdot = p.tdot;
        u3.iupdate = p.iupdate;
        u3.iuphard = p.iuphard;
        u3.vlast = vlast;
        K("k_upd3", [&] { launch_upd3(d, u3, st); });
        // averages that only depend on host values
        double vsym[9];
        sym33(velgradavg, vsym);
        lvmavg = vm_strain(velgradavg);
        dvmavg = vm_strain(vsym);
        evmavg = evmavg + dvmavg * p.tdot;
        const double Lref = std::max(lvmavg, EVP_TINY);
        K("k_diag", [&] { launch_diag(d, std::max(1.0e-12 * Lref, EVP_TINY), st); });
        // time bookkeeping and the tdot ramp are host-only; they fix the tdot calc_c0 sees.  The
        // VTK "last step" test uses the step count from before the ramp, as the reference
        // writes its fields before ramping (LS-EVPFFT.f90:525-535, then 557-581).
        es.nsteps_written = p.nsteps;
        es.tdot_used = p.tdot;
        es.tdotref_used = p.tdotref;
        if (p.ictrl == -1) {
            proc_time_done += es.tdot_used;
            p.tdot = tdot_plan;
        }
        sim_time += es.tdot_used;
        if (p.ictrl == -1) {
            if (tdot_plan < p.tdotref && nconverged >= 5) {
                nconverged = 0;
                tdot_plan = std::min(2.0 * tdot_plan, p.tdotref);
                const double remaining = std::max(0.0, proc_time_target - proc_time_done);
                const int left = (int)std::ceil(remaining / tdot_plan);
                const int nnew = imicro + left;
                total_macrosteps += nnew - p.nsteps;
                p.nsteps = nnew;
                p.tdot = (remaining > 0.0) ? std::min(tdot_plan, remaining) : tdot_plan;
            }
        } else if (p.tdot < p.tdotref && nconverged >= 5) {
            nconverged = 0;
            const double tdot = p.tdot;
            p.tdot = std::min(2.0 * p.tdot, p.tdotref);
            int left = p.nsteps - imicro;
            left = (int)std::ceil((double)left * tdot / p.tdot);
            total_macrosteps += left - (p.nsteps - imicro);
            p.nsteps = imicro + left;
        }
        es.conv_for_count = did_converge;
        K("k_c0", [&] { launch_c0(d, p.tdot, p.tdotref, st); });
        CK(cudaGetLastError());
        CK(cudaEventRecord(ev1, st));
        fetch_red_async();
    }

    void end_finish() {
        check_red();
        ProcessData& p = P();
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, ev0, ev1) == cudaSuccess) gpu_ms += ms;
        // update_defgrad averages (host side of various_functions.f90:2250-2266)
        const double* u1o = h_red + OFF_UPD1;
        edotvmmx = u1o[39];
        if (p.iupdate == 1) {
            const double dav = u1o[38];
            for (int c = 0; c < 9; c++) { defgradavg[c] = u1o[c]; dinvc[c] = u1o[9 + c] / dav; }
            wphcsol = u1o[36] / dav;
            wphcgas = u1o[37] / dav;
            for (int c = 0; c < 9; c++) dinvcs[c] = u1o[18 + c] / dav / wphcsol;
            if (wphcgas > 0.0) for (int c = 0; c < 9; c++) dinvcg[c] = u1o[27 + c] / dav / wphcgas;
            else for (int c = 0; c < 9; c++) dinvcg[c] = (c % 4 == 0) ? 1.0 : 0.0;
        }
        // macro averages (LS-EVPFFT.f90:465-523)
        const double* r3 = h_red + OFF_UPD3;
        double ep6[6], ea6[6], el6[6], ed6[6], ss6[6];
        for (int c = 0; c < 6; c++) {
            ep6[c] = r3[c] / wphcsol;
            ea6[c] = r3[6 + c] / wphcsol;
            ed6[c] = r3[12 + c] / wphcsol;
            ss6[c] = r3[18 + c] / wphcsol;
            // eelavg = eavg + (disgradsym - ept) * wgtc of the last solid voxel (LS-EVPFFT.f90:482-483)
            el6[c] = (r3[6 + c] + (r3[30 + c] - r3[36 + c]) * r3[42]) / wphcsol;
        }
        s6_to_t2(ep6, epavg); s6_to_t2(ea6, eavg); s6_to_t2(el6, eelavg); s6_to_t2(ed6, edotpavg); s6_to_t2(ss6, sgsolavg);
        const double nsolid = r3[25], nsys_solid = r3[27];
        const double gammaavg = nsolid > 0.0 ? r3[24] / nsolid : 0.0;
        const double gavg = nsys_solid > 0.0 ? r3[26] / nsys_solid : 0.0;
        const double geffavg = r3[28] > 0.0 ? r3[29] / r3[28] : gavg;
        evmpavg = vm_strain(epavg);
        dvmpavg = vm_strain(edotpavg);
        if (p.iwfields == 1) {
            const int aw = std::abs(p.iwstep);
            const bool due = (aw != 0 && imicro % aw == 0) || (p.iwstep < 0 && imicro == es.nsteps_written);
            if (due && write_vtk_files) write_vtk(imacroloop);
        }
        finish_diag();
        dg.erre = erre; dg.errs = errs; dg.errsbc = errsbc;
        dg.tdotref = es.tdotref_used;
        dg.s33_target = p.scauchy[8];
        dg.s33 = sgavg[8];
        dg.s33_sol = sgsolavg[8];
        dg.devm_inc_max = edotvmmx * es.tdot_used;
        wall_time = (double)(std::time(nullptr) - start);
        write_rows(es.iter_done, imacroloop, ipr, sim_time, wall_time, es.tdot_used, dg.tdotref, gammaavg, gavg, geffavg);
        if (es.conv_for_count) nconverged++;
        finish_c0(p);
        imacroloop++;
        macrosteps_done++;
    }

    // ------------------------------------------------------------ round length
    // The host looks at the event codes after each round of queued iterations.  A solve expects
    // its increment to take as many iterations as the previous one did, so a round ends where
    // that expectation runs out instead of after a fixed count: a member that converges does not
    // sit through the rest of a long round, and one far from convergence is not polled often.
    int prev_inc_iters = 0;  // iterations of the previous increment (0: none yet)
    int inc_launched = 0;    // iterations queued in this increment (since its last restart)
    int want_iters() const {
        if (prev_inc_iters <= 0) return 4;
        const int rem = prev_inc_iters - inc_launched;
        return rem > 0 ? rem : 2;  // past the expectation: look every two iterations
    }

    // ------------------------------------------------------------ one macrostep of a solve on its own
    // The engine of one member runs the increment's iterations in rounds (round_length); the host
    // looks at the control block between rounds (events: convergence, ITMAX, errors).
    std::unique_ptr<Engine> solo;
    bool macrostep() {
        if (!begin_increment()) return false;
        if (!solo) {
            solo.reset(new Engine(st));
            solo->set_members({Engine::Member{entry(), modal ? 1 : 0, prec}});
        } else {
            solo->update_entry(0, entry());
        }
        Engine::Timer timer = [this](const char* name, const std::function<void()>& f) { K(name, f); };
        const int per_iter = solo->launches_per_iteration();
        long long queued = 0;
        while (true) {
            check_deadline();
            const int k = round_length(want_iters());
            if ((queued += k) > 100000 + 2 * kMaxRound) throw SolveError("equilibrium iteration did not converge", -4);
            solo->launch(k, profile ? &timer : nullptr);
            inc_launched += k;
            if (!profile) launches += (long long)k * per_iter;
            const int ev = solo->read_events()[0];
            if (ev == EV_RUNNING) continue;
            pull_ctl();
            if (handle_event(ev)) break;
            solo->update_entry(0, entry());
        }
        end_launch();
        sync();
        end_finish();
        return true;
    }

    void finish_diag() {
        const double* r = h_red + OFF_DIAG;
        const long long n1 = d.n1, n2 = d.n2;
        dg.dl_rms = r[1] > 0 ? std::sqrt(r[0] / r[1]) : 0.0;
        dg.dl_rms_sol = r[3] > 0 ? std::sqrt(r[2] / r[3]) : 0.0;
        dg.dl_rms_gas = r[5] > 0 ? std::sqrt(r[4] / r[5]) : 0.0;
        dg.dl_max = r[6]; dg.dl_max_sol = r[7]; dg.dl_max_gas = r[8];
        dg.volinc_sol = r[9]; dg.volinc_gas = r[10]; dg.rot_sol = r[11]; dg.rot_gas = r[12];
        dg.stretch_sol = r[13]; dg.stretch_gas = r[14];
        dg.cond_sol = r[15]; dg.cond_gas = r[16]; dg.cond_cgas = r[17];
        dg.detF_min = -r[18];
        auto idx = [&](double vv, int* out) {
            if (vv < 0) { out[0] = out[1] = out[2] = 0; return; }
            long long v = (long long)vv;
            out[0] = (int)(v % n1) + 1; out[1] = (int)((v / n1) % n2) + 1; out[2] = (int)(v / (n1 * n2)) + 1;
        };
        dg.detF_min_sol = r[19];
        idx(r[20], dg.imin_sol);
        dg.detF_min_gas = r[21];
        idx(r[22], dg.imin_gas);
        if (dg.detF_min >= EVP_HUGE * 0.5) dg.detF_min = 0.0;
        if (dg.detF_min_sol >= EVP_HUGE * 0.5) dg.detF_min_sol = 0.0;
        if (dg.detF_min_gas >= EVP_HUGE * 0.5) dg.detF_min_gas = 0.0;
        dg.dvelgradavg_mag = frob3(dvelgradavg);
        dg.detF_min_prev = dg.detF_min;
        dg.detF_min_sol_rel = safe_rel(dg.detF_min_sol, dg.detF_min_sol_prev);
        dg.detF_min_sol_prev = dg.detF_min_sol;
        dg.detF_min_gas_rel = safe_rel(dg.detF_min_gas, dg.detF_min_gas_prev);
        dg.detF_min_gas_prev = dg.detF_min_gas;
        dg.volinc_sol_rel = safe_rel(dg.volinc_sol, dg.volinc_sol_prev); dg.volinc_sol_prev = dg.volinc_sol;
        dg.volinc_gas_rel = safe_rel(dg.volinc_gas, dg.volinc_gas_prev); dg.volinc_gas_prev = dg.volinc_gas;
        dg.stretch_sol_rel = safe_rel(dg.stretch_sol, dg.stretch_sol_prev); dg.stretch_sol_prev = dg.stretch_sol;
        dg.stretch_gas_rel = safe_rel(dg.stretch_gas, dg.stretch_gas_prev); dg.stretch_gas_prev = dg.stretch_gas;
    }

    void finish_c0(const ProcessData& p) {  // calc_c0 tail (various_functions.f90:2633-2647)
        const double* r = h_red + OFF_C0;
        double dP[36], a[36], ai[36];
        for (int c = 0; c < 36; c++) a[c] = r[c] / wphcsol;  // <dsg/de> in the b-basis
        for (int c = 0; c < 36; c++) dP[c] = r[36 + c] / wphsol;
        std::memcpy(ai, a, sizeof(a));
        if (lu_inverse(ai, 6) != 0) throw SolveError("Singular matrix in lu_inverse (calc_c0)", -3);
        b66_to_t4(ai, de_ds);
        for (int c = 0; c < 36; c++) { c066[c] = dP[c] * p.xc0; a[c] = dP[c] * p.xc0; }
        if (lu_inverse(a, 6) != 0) throw SolveError("Singular matrix in lu_inverse (calc_c0)", -3);
        b66_to_t4(c066, c0);
        b66_to_t4(a, s0);
        upload_c0();
    }

    // ------------------------------------------------------------ outputs
    std::string csv_path(const char* name) const {
        if (!outdir.empty() && outdir.back() == '/') return outdir + name;
        return outdir + "/" + name;
    }
    void write_headers() {
        FILE* f = std::fopen(csv_path("diagnostics.csv").c_str(), "w");
        if (!f) throw SolveError("write_diagnostics: failed to open diagnostics.csv for writing", -5);
        std::fputs("iter,macrostep,ipr,sim_time,wall_time,tdot,vm_max_inc,tdotref,erre,errs,errsbc,s33_target,s33,s33_sol,"
                   "detF_min_sol,detF_min_gas,detF_min_sol_rel,detF_min_gas_rel,volinc_max_sol,volinc_max_gas,volinc_max_sol_rel,"
                   "volinc_max_gas_rel,stretchinc_max_sol,stretchinc_max_gas,stretchinc_max_sol_rel,stretchinc_max_gas_rel,"
                   "rotang_max_sol,rotang_max_gas,dL_step_rms_sol,dL_step_rms_gas,dL_step_rms,dL_step_max_sol,dL_step_max_gas,"
                   "dL_step_max,dvelgradavg_mag,cond_c066mod_max_sol,cond_c066mod_max_gas,cond_cgas_max,imin_sol_i,imin_sol_j,"
                   "imin_sol_k,imin_gas_i,imin_gas_j,imin_gas_k\n", f);
        std::fclose(f);
        f = std::fopen(csv_path("results.csv").c_str(), "w");
        if (!f) throw SolveError("results: failed to open results.csv for writing", -5);
        std::fputs("iter,macrostep,ipr,sim_time,wall_time,tdot,tdot_ref,eav11,eav22,eav33,eav23,eav13,eav12,sav11,sav22,sav33,"
                   "sav23,sav13,sav12,epav11,epav22,epav33,epav23,epav13,epav12,eelav11,eelav22,eelav33,eelav23,eelav13,"
                   "eelav12,vgrad11,vgrad22,vgrad33,vgrad23,vgrad13,vgrad12,edotp11,edotp22,edotp33,edotp23,edotp13,edotp12,"
                   "evm,evmp,dvm,dvmp,svm,gamma,g,geff\n", f);
        std::fclose(f);
    }
    void write_rows(int it, int imac, int ip, double st_, double wt, double tdot, double tdotref, double gamma, double g, double geff) {
        double* R = last_results;
        int c = 0;
        R[c++] = it; R[c++] = imac; R[c++] = ip; R[c++] = st_; R[c++] = wt; R[c++] = tdot; R[c++] = tdotref;
        auto put6 = [&](const double* m) { R[c++] = m[0]; R[c++] = m[4]; R[c++] = m[8]; R[c++] = m[5]; R[c++] = m[2]; R[c++] = m[1]; };
        put6(eavg); put6(sgsolavg); put6(epavg); put6(eelavg); put6(velgradavg); put6(edotpavg);
        R[c++] = evmavg; R[c++] = evmpavg; R[c++] = dvmavg; R[c++] = dvmpavg; R[c++] = svmavg; R[c++] = gamma; R[c++] = g; R[c++] = geff;
        double D[44] = {(double)it, (double)imac, (double)ip, st_, wt, tdot, dg.devm_inc_max, dg.tdotref, dg.erre, dg.errs, dg.errsbc,
                        dg.s33_target, dg.s33, dg.s33_sol, dg.detF_min_sol, dg.detF_min_gas, dg.detF_min_sol_rel, dg.detF_min_gas_rel,
                        dg.volinc_sol, dg.volinc_gas, dg.volinc_sol_rel, dg.volinc_gas_rel, dg.stretch_sol, dg.stretch_gas,
                        dg.stretch_sol_rel, dg.stretch_gas_rel, dg.rot_sol, dg.rot_gas, dg.dl_rms_sol, dg.dl_rms_gas, dg.dl_rms,
                        dg.dl_max_sol, dg.dl_max_gas, dg.dl_max, dg.dvelgradavg_mag, dg.cond_sol, dg.cond_gas, dg.cond_cgas,
                        (double)dg.imin_sol[0], (double)dg.imin_sol[1], (double)dg.imin_sol[2], (double)dg.imin_gas[0],
                        (double)dg.imin_gas[1], (double)dg.imin_gas[2]};
        std::memcpy(last_diag, D, sizeof(D));
        if (!write_files) return;
        std::string line;
        for (int q = 0; q < 44; q++) {
            line += (q < 3 || q >= 38) ? std::to_string((long long)D[q]) : g0(D[q]);
            line += (q == 43) ? '\n' : ',';
        }
        FILE* f = std::fopen(csv_path("diagnostics.csv").c_str(), "a");
        if (!f) throw SolveError("write_diagnostics: failed to open diagnostics.csv for append", -5);
        std::fputs(line.c_str(), f);
        std::fclose(f);
        line.clear();
        for (int q = 0; q < 51; q++) {
            line += (q < 3) ? std::to_string((long long)R[q]) : g0(R[q]);
            line += (q == 50) ? '\n' : ',';
        }
        f = std::fopen(csv_path("results.csv").c_str(), "a");
        if (!f) throw SolveError("write_results: failed to open results.csv for append", -5);
        std::fputs(line.c_str(), f);
        std::fclose(f);
    }

    std::vector<double> field_host(double* dp, size_t n) {
        std::vector<double> h(n);
        CK(cudaMemcpyAsync(h.data(), dp, n * sizeof(double), cudaMemcpyDeviceToHost, st));
        d2h += (long long)(n * sizeof(double));
        sync();
        return h;
    }
    // Lines [0, n) of one VTK block, formatted by line(buffer, index) on several host threads in
    // contiguous slices and written in order: the file is byte-identical to a serial write.
    template <class Line>
    static void emit_lines(FILE* f, long long n, Line&& line) {
        const long long per = 16384;  // lines per slice (~1 MB of text)
        const long long nslice = (n + per - 1) / per;
        const int nthr = (int)std::max(1LL, std::min<long long>(nslice, std::max(1u, std::thread::hardware_concurrency())));
        const long long wave = (long long)nthr;
        std::vector<std::string> buf(nthr);
        for (long long s0 = 0; s0 < nslice; s0 += wave) {
            const int m = (int)std::min(wave, nslice - s0);
            auto work = [&](int t) {
                std::string& o = buf[t];
                o.clear();
                const long long a = (s0 + t) * per, b = std::min(n, a + per);
                for (long long i = a; i < b; i++) line(o, i);
            };
            std::vector<std::thread> th;
            for (int t = 1; t < m; t++) th.emplace_back(work, t);
            work(0);
            for (auto& x : th) x.join();
            for (int t = 0; t < m; t++) std::fwrite(buf[t].data(), 1, buf[t].size(), f);
        }
    }

    // write_vtk_cell (IO_functions.f90:945-1235): the fields are copied to the host here, in the
    // solve's stream order; the text is formatted and written by vtk_file, in the background when
    // async_vtk is set.
    void write_vtk(int istp) {
        wait_vtk();
        const long long N = d.N;
        const int n1 = d.n1, n2 = d.n2, n3 = d.n3;
        VtkFields v;
        v.xn = field_host(d.xnode, 3 * (size_t)(n1 + 1) * (n2 + 1) * d.n3node);
        v.gd = field_host(d.gamdot, (size_t)d.nsys * N);
        v.ga = field_host(d.gacumgr, N);
        v.fp = field_host(d.Fp, 9 * N);
        v.sg = field_host(d.sg, 6 * N);
        v.F = field_host(d.F, 9 * N);
        v.dF = field_host(d.detF, N);
        v.ep = field_host(d.epvm, N);
        v.vg = field_host(d.velgrad, 9 * N);
        char name[64];
        std::snprintf(name, sizeof(name), "microstr_cell_fields_stp_%05d.vtk", istp);
        auto job = [this, path = outdir + "/" + name, v = std::move(v)]() { vtk_file(path, v); };
        if (async_vtk) vtk_job = std::async(std::launch::async, std::move(job));
        else job();
    }
    struct VtkFields {
        std::vector<double> xn, gd, ga, fp, sg, F, dF, ep, vg;
    };
    // the file itself, from host copies and the deck's grain and phase ids (read-only here)
    void vtk_file(const std::string& path, const VtkFields& v) const {
        const long long N = d.N;
        const int n1 = d.n1, n2 = d.n2, n3 = d.n3;
        const std::vector<double>&xn = v.xn, &gd = v.gd, &ga = v.ga, &fp = v.fp, &sg = v.sg, &F = v.F, &dF = v.dF,
                                   &ep = v.ep, &vg = v.vg;
        FILE* f = std::fopen(path.c_str(), "w");
        if (!f) throw SolveError("ioerr in writevtk", -5);
        char b[256];
        auto put = [&](const char* text) { std::fputs(text, f); };
        put("# vtk DataFile Version 3.0\nmicrostructure data\nASCII\nDATASET UNSTRUCTURED_GRID\n");
        const long long nn1 = n1 + 1, nn2 = n2 + 1;
        auto nid = [&](long long i, long long j, long long k) { return i + nn1 * (j + nn2 * k); };
        auto point = [&](std::string& o, long long q) {  // node q in (i, j, k) order, i fastest
            put_e18(o, xn[3 * q]);
            put_e18(o, xn[3 * q + 1]);
            put_e18(o, xn[3 * q + 2]);
            o += '\n';
        };
        long long ncell;
        if (n3 == 1) {
            std::snprintf(b, sizeof(b), "POINTS%10lld double\n", nn1 * nn2);
            put(b);
            emit_lines(f, nn1 * nn2, point);
            ncell = (long long)n1 * n2;
            std::snprintf(b, sizeof(b), "CELLS%10lld%10lld\n", ncell, ncell * 5);
            put(b);
            emit_lines(f, ncell, [&](std::string& o, long long c) {
                char t[128];
                const long long i = c % n1, j = c / n1;
                std::snprintf(t, sizeof(t), "%10d%10lld%10lld%10lld%10lld\n", 4, nid(i, j, 0), nid(i + 1, j, 0), nid(i, j + 1, 0),
                              nid(i + 1, j + 1, 0));
                o += t;
            });
            std::snprintf(b, sizeof(b), "CELL_TYPES%10lld\n", ncell);
            put(b);
            emit_lines(f, ncell, [](std::string& o, long long) { o += "    8\n"; });
        } else {
            std::snprintf(b, sizeof(b), "POINTS%10lld double\n", nn1 * nn2 * (n3 + 1));
            put(b);
            emit_lines(f, nn1 * nn2 * (n3 + 1), point);
            ncell = N;
            std::snprintf(b, sizeof(b), "CELLS%10lld%10lld\n", ncell, ncell * 9);
            put(b);
            emit_lines(f, ncell, [&](std::string& o, long long c) {
                char t[160];
                const long long i = c % n1, j = (c / n1) % n2, k = c / ((long long)n1 * n2);
                std::snprintf(t, sizeof(t), "%10d%10lld%10lld%10lld%10lld%10lld%10lld%10lld%10lld\n", 8, nid(i, j, k), nid(i + 1, j, k),
                              nid(i + 1, j + 1, k), nid(i, j + 1, k), nid(i, j, k + 1), nid(i + 1, j, k + 1), nid(i + 1, j + 1, k + 1),
                              nid(i, j + 1, k + 1));
                o += t;
            });
            std::snprintf(b, sizeof(b), "CELL_TYPES%10lld\n", ncell);
            put(b);
            emit_lines(f, ncell, [](std::string& o, long long) { o += "   12\n"; });
        }
        std::snprintf(b, sizeof(b), "CELL_DATA%10lld\nFIELD FieldData%10d\n", ncell, 11);
        put(b);
        const int ns = d.nsys;
        std::snprintf(b, sizeof(b), "gamdot%3d%10lld double\n", ns, ncell);
        put(b);
        emit_lines(f, N, [&](std::string& o, long long v) {
            for (int q = 0; q < ns; q++) put_e18(o, gd[q * N + v]);
            o += '\n';
        });
        auto scalar = [&](const char* nm, const std::vector<double>& a) {
            std::snprintf(b, sizeof(b), "%s%3d%10lld double\n", nm, 1, ncell);
            put(b);
            emit_lines(f, N, [&](std::string& o, long long v) {
                put_e18(o, a[v]);
                o += '\n';
            });
        };
        auto tens9 = [&](const char* nm, const std::vector<double>& a) {  // column-major order
            std::snprintf(b, sizeof(b), "%s%3d%10lld double\n", nm, 9, ncell);
            put(b);
            emit_lines(f, N, [&](std::string& o, long long v) {
                for (int c = 0; c < 3; c++)
                    for (int r = 0; r < 3; r++) put_e18(o, a[(3 * r + c) * N + v]);
                o += '\n';
            });
        };
        scalar("gamdot_acum", ga);
        tens9("def_grad_p", fp);
        std::snprintf(b, sizeof(b), "stress%3d%10lld double\n", 6, ncell);
        put(b);
        emit_lines(f, N, [&](std::string& o, long long v) {
            put_e18(o, sg[0 * N + v]); put_e18(o, sg[1 * N + v]); put_e18(o, sg[2 * N + v]);
            put_e18(o, sg[5 * N + v]); put_e18(o, sg[3 * N + v]); put_e18(o, sg[4 * N + v]);
            o += '\n';
        });
        std::vector<double> svm(N);
        for (long long v = 0; v < N; v++) {
            double s6[6], t[9];
            for (int c = 0; c < 6; c++) s6[c] = sg[c * N + v];
            s6_to_t2(s6, t);
            svm[v] = vm_stress(t);
        }
        scalar("svm", svm);
        tens9("def_grad", F);
        scalar("det_def_grad", dF);
        std::snprintf(b, sizeof(b), "gr_id%3d%10lld int\n", 1, ncell);
        put(b);
        emit_lines(f, N, [&](std::string& o, long long v) {
            char t[32];
            std::snprintf(t, sizeof(t), "%10d\n", dk.grain[v]);
            o += t;
        });
        std::snprintf(b, sizeof(b), "ph_id%3d%10lld int\n", 1, ncell);
        put(b);
        emit_lines(f, N, [&](std::string& o, long long v) {
            char t[32];
            std::snprintf(t, sizeof(t), "%10d\n", dk.phase_id[v]);
            o += t;
        });
        scalar("epvm", ep);
        tens9("velgrad", vg);
        std::fclose(f);
    }

    long long get_field(const std::string& name, double* out, long long cap) {
        const long long N = d.N;
        const int ns = d.nsys;
        auto soa_to_aos = [&](double* dp, int ncomp, const int* map, int nout) -> long long {
            if ((long long)nout * N > cap) return -1;
            auto h = field_host(dp, (size_t)ncomp * N);
            for (long long v = 0; v < N; v++)
                for (int c = 0; c < nout; c++) out[nout * v + c] = h[(size_t)map[c] * N + v];
            return (long long)nout * N;
        };
        static const int id9[9] = {0, 1, 2, 3, 4, 5, 6, 7, 8};
        static const int s6to9[9] = {0, 5, 4, 5, 1, 3, 4, 3, 2};  // (11,22,33,23,13,12) -> row-major 3x3
        if (name == "sg") return soa_to_aos(d.sg, 6, s6to9, 9);
        if (name == "sgt") return soa_to_aos(d.sgt, 6, s6to9, 9);
        if (name == "edotp") return soa_to_aos(d.edotp, 6, s6to9, 9);
        if (name == "ept") return soa_to_aos(d.ept, 6, s6to9, 9);
        if (name == "disgradsym") return soa_to_aos(d.disgradsym, 6, s6to9, 9);
        if (name == "velgrad") return soa_to_aos(d.velgrad, 9, id9, 9);
        if (name == "velgradold") return soa_to_aos(d.velgradold, 9, id9, 9);
        if (name == "dvelgradref") return soa_to_aos(d.dvr, 9, id9, 9);
        if (name == "defgrad") return soa_to_aos(d.F, 9, id9, 9);
        if (name == "defgradinv") return soa_to_aos(d.Finv, 9, id9, 9);
        if (name == "defgrade") return soa_to_aos(d.Fe, 9, id9, 9);
        if (name == "defgradp") return soa_to_aos(d.Fp, 9, id9, 9);
        if (name == "detF") return soa_to_aos(d.detF, 1, id9, 1);
        if (name == "wgtc") return soa_to_aos(d.wgtc, 1, id9, 1);
        if (name == "gacumgr") return soa_to_aos(d.gacumgr, 1, id9, 1);
        if (name == "epvm") return soa_to_aos(d.epvm, 1, id9, 1);
        std::vector<int> m(72);
        for (int c = 0; c < 72; c++) m[c] = c;
        if (name == "gamdot") return soa_to_aos(d.gamdot, ns, m.data(), ns);
        if (name == "crss") return soa_to_aos(d.crss, 2 * ns, m.data(), 2 * ns);
        if (name == "trialtau") return soa_to_aos(d.trialtau, 2 * ns, m.data(), 2 * ns);
        if (name == "sch") return soa_to_aos(d.sch, 5 * ns, m.data(), 5 * ns);
        if (name == "c066mod") return soa_to_aos(d.c066mod, 36, m.data(), 36);
        if (name == "sg66") return soa_to_aos(d.sg66, 36, m.data(), 36);
        if (name == "macro") {  // c066, c0, s0, de_ds (reference-medium state, host copies)
            if (cap < 279) return -1;
            std::memcpy(out, c066, sizeof(c066));
            std::memcpy(out + 36, c0, sizeof(c0));
            std::memcpy(out + 117, s0, sizeof(s0));
            std::memcpy(out + 198, de_ds, sizeof(de_ds));
            return 279;
        }
        if (name == "xnode") {
            long long n = 3LL * (d.n1 + 1) * (d.n2 + 1) * d.n3node;
            if (n > cap) return -1;
            CK(cudaMemcpyAsync(out, d.xnode, n * sizeof(double), cudaMemcpyDeviceToHost, st));
            sync();
            return n;
        }
        return -2;
    }
};

// ------------------------------------------------------------ a batch of solves (evp_batch.h)
class Batch {
public:
    struct Slot {
        std::unique_ptr<Solver> s;
        int state = 0;  // 0 running, 1 finished
        int status = 0;
        std::string err;
        evp_report rep{};
        std::chrono::steady_clock::time_point t0;
    };
    cudaStream_t st = nullptr;
    std::unique_ptr<Engine> eng;
    std::vector<Slot> slots;  // slot ids stay valid; a removed slot keeps its record, not its solver
    std::vector<int> members;  // running slots, in the engine's member order
    bool dirty = false;
    int round_k = 0;  // iterations of the round in flight

    cudaEvent_t round_ev = nullptr;  // recorded after a launched round's iterations
    bool in_round = false;

    // priority: CUDA stream priority of the batch's stream (0 default; lower numbers run first)
    explicit Batch(int priority = 0) {
        CK(cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, priority));
        CK(cudaEventCreateWithFlags(&round_ev, cudaEventDisableTiming));
        eng.reset(new Engine(st));
    }
    ~Batch() {
        if (round_ev) cudaEventDestroy(round_ev);
        eng.reset();
        for (auto& sl : slots) sl.s.reset();
        if (st) {
            cudaStreamSynchronize(st);
            cudaStreamDestroy(st);
        }
    }

    void finish(int id, int status, const std::string& err) {
        Slot& sl = slots[id];
        if (sl.state == 1) return;
        std::string e = err;
        if (sl.s) {  // the member's last VTK file is complete before it is reported done
            try {
                sl.s->wait_vtk();
            } catch (SolveError& x) {
                if (status == 0) {
                    status = x.code;
                    e = x.what();
                }
            } catch (std::exception& x) {
                if (status == 0) {
                    status = -1;
                    e = x.what();
                }
            }
        }
        sl.state = 1;
        sl.status = status;
        sl.err = e;
        std::memset(&sl.rep, 0, sizeof(sl.rep));
        if (sl.s) {
            Solver& s = *sl.s;
            sl.rep.macrosteps = s.macrosteps_done;
            sl.rep.equilibrium_iters = s.total_iters;
            sl.rep.voxel_iters = s.total_iters * s.d.N;
            sl.rep.n1 = s.d.n1;
            sl.rep.n2 = s.d.n2;
            sl.rep.n3 = s.d.n3;
            sl.rep.h2d_bytes = s.h2d;
            sl.rep.d2h_bytes = s.d2h;
        }
        sl.rep.status = status;
        sl.rep.wall_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - sl.t0).count();
        dirty = true;
    }

    int add(Deck&& dk, const std::string& fft_in, const std::string& out, int mix, int modal, int flags, double deadline_s,
            std::string& err) {
        const int id = (int)slots.size();
        slots.emplace_back();
        slots[id].t0 = std::chrono::steady_clock::now();
        slots[id].s.reset(new Solver());
        Solver& s = *slots[id].s;
        s.async_vtk = true;  // a member's files are needed when it finishes (finish waits for them)
        try {
            s.open(fft_in, out, mix, modal, flags & ~EVP_PROFILE, st, &dk);
            if (deadline_s > 0.0) {
                s.has_deadline = true;
                s.deadline = slots[id].t0 + std::chrono::duration_cast<std::chrono::steady_clock::duration>(
                                                std::chrono::duration<double>(deadline_s));
            }
            if (!s.begin_increment()) {
                finish(id, 0, "");
                return id;
            }
        } catch (SolveError& e) {
            err = e.what();
            finish(id, e.code, err);
            slots[id].s.reset();
            return id;
        } catch (std::exception& e) {
            err = e.what();
            finish(id, -1, err);
            slots[id].s.reset();
            return id;
        }
        dirty = true;
        return id;
    }

    void rebuild() {
        members.clear();
        std::vector<Engine::Member> m;
        for (int id = 0; id < (int)slots.size(); id++) {
            if (slots[id].state != 0 || !slots[id].s) continue;
            members.push_back(id);
            Solver& s = *slots[id].s;
            m.push_back(Engine::Member{s.entry(), s.modal ? 1 : 0, s.prec});
        }
        eng->set_members(m);
        dirty = false;
    }

    // One round: a few iterations of every running member (launch_round, asynchronous), then,
    // once they have run (round_done), the host side of their events (finish_round).  The round
    // is as long as the member expected to stop first wants (round_length).
    bool launch_round() {
        if (in_round) return true;
        if (dirty) rebuild();
        if (members.empty()) return false;
        int want = 1 << 30;
        for (int id : members)
            if (slots[id].s && slots[id].state == 0) want = std::min(want, slots[id].s->want_iters());
        round_k = round_length(want);
        eng->launch(round_k, nullptr);
        for (int id : members)
            if (slots[id].s && slots[id].state == 0) slots[id].s->inc_launched += round_k;
        CK(cudaEventRecord(round_ev, st));
        in_round = true;
        return true;
    }
    bool round_done() const { return !in_round || cudaEventQuery(round_ev) != cudaErrorNotReady; }
    void round() {
        if (launch_round()) finish_round();
    }
    void finish_round() {
        if (!in_round) return;
        in_round = false;
        const int per_iter = eng->launches_per_iteration();
        const int* ev = eng->read_events();
        std::vector<int> ended;  // member positions whose increment iteration is over
        for (int i = 0; i < (int)members.size(); i++) {
            const int id = members[i];
            if (!slots[id].s || slots[id].state != 0) continue;
            Solver& s = *slots[id].s;
            s.launches += (long long)round_k * per_iter;
            try {
                s.check_deadline();
                if (ev[i] == EV_RUNNING) continue;
                s.pull_ctl();
                if (s.handle_event(ev[i])) ended.push_back(i);
                else eng->update_entry(i, s.entry());
            } catch (SolveError& e) {
                finish(id, e.code, e.what());
            } catch (std::exception& e) {
                finish(id, -1, e.what());
            }
        }
        std::vector<int> launched;
        for (int i : ended) {
            const int id = members[i];
            if (slots[id].state != 0) continue;
            try {
                slots[id].s->end_launch();
                launched.push_back(i);
            } catch (SolveError& e) {
                finish(id, e.code, e.what());
            }
        }
        if (!launched.empty()) CK(cudaStreamSynchronize(st));
        for (int i : launched) {
            const int id = members[i];
            Solver& s = *slots[id].s;
            try {
                s.end_finish();
                if (!s.begin_increment()) finish(id, 0, "");
                else eng->update_entry(i, s.entry());
            } catch (SolveError& e) {
                finish(id, e.code, e.what());
            } catch (std::exception& e) {
                finish(id, -1, e.what());
            }
        }
    }

    int running() const {
        int n = 0;
        for (auto& sl : slots) n += (sl.state == 0 && sl.s) ? 1 : 0;
        return n;
    }
};

Batch* batch_create(int priority) { return new Batch(priority); }
bool batch_launch(Batch* b) { return b->launch_round(); }
bool batch_ready(Batch* b) { return b->round_done(); }
int batch_finish(Batch* b) {
    b->finish_round();
    if (b->dirty) b->rebuild();
    return b->running();
}
int batch_priority_range(int* lowest) {
    int lo = 0, hi = 0;
    cudaDeviceGetStreamPriorityRange(&lo, &hi);
    if (lowest) *lowest = lo;
    return hi;  // the highest priority (numerically smallest)
}
void batch_destroy(Batch* b) { delete b; }
int batch_add(Batch* b, Deck&& dk, const std::string& fft_in, const std::string& out_dir, int mix, int modal, int flags,
              double deadline_s, std::string& err) {
    return b->add(std::move(dk), fft_in, out_dir, mix, modal, flags, deadline_s, err);
}
int batch_step(Batch* b, int rounds) {
    for (int r = 0; r < rounds; r++) {
        b->round();
        if (b->running() == 0) break;
    }
    if (b->dirty) b->rebuild();
    return b->running();
}
int batch_slot(Batch* b, int slot, int* status, evp_report* rep, std::string* err) {
    if (slot < 0 || slot >= (int)b->slots.size()) return -1;
    const Batch::Slot& sl = b->slots[slot];
    if (status) *status = sl.status;
    if (rep) *rep = sl.rep;
    if (err) *err = sl.err;
    return sl.state;
}
void batch_remove(Batch* b, int slot) {
    if (slot < 0 || slot >= (int)b->slots.size()) return;
    Batch::Slot& sl = b->slots[slot];
    if (sl.state == 0) {
        b->finish(slot, -7, "removed while running");
    }
    sl.s.reset();
    b->dirty = true;
}
int batch_running(Batch* b) { return b->running(); }

}  // namespace evp

using evp::SolveError;
using evp::Solver;

struct evp_solve {
    Solver s;
};

static int fail(const std::string& m, int code) {
    evp::g_last_error = m;
    return code;
}

extern "C" {

int evp_version(void) { return 1; }

const char* evp_last_error(void) { return evp::g_last_error.c_str(); }

// async_vtk: VTK files (the step-0 one included) written in the background, finished by wait_vtk
static int open_solve(const char* fft_in, const char* out_dir, int mix, int modal, int flags, bool async_vtk,
                      evp_solve** out) {
    if (!fft_in || !out) return fail("evp_open: null argument", -7);
    *out = nullptr;
    evp_solve* h = new evp_solve();
    h->s.async_vtk = async_vtk;
    try {
        h->s.open(fft_in, out_dir ? out_dir : "", mix, modal, flags);
    } catch (SolveError& e) {
        delete h;
        return fail(e.what(), e.code);
    } catch (std::exception& e) {
        delete h;
        return fail(e.what(), -1);
    }
    *out = h;
    return 0;
}

int evp_open(const char* fft_in, const char* out_dir, int mix, int modal, int flags, evp_solve** out) {
    return open_solve(fft_in, out_dir, mix, modal, flags, false, out);
}

int evp_advance(evp_solve* h, int nmacro, int* done) {
    if (!h) return fail("evp_advance: null handle", -7);
    int n = 0;
    try {
        for (int i = 0; i < nmacro; i++) {
            if (!h->s.macrostep()) break;
            n++;
        }
    } catch (SolveError& e) {
        if (done) *done = n;
        return fail(e.what(), e.code);
    } catch (std::exception& e) {
        if (done) *done = n;
        return fail(e.what(), -1);
    }
    if (done) *done = n;
    return 0;
}

int evp_get_field(evp_solve* h, const char* name, double* host_out, long long capacity, long long* written) {
    if (!h || !name || !host_out) return fail("evp_get_field: null argument", -7);
    try {
        long long n = h->s.get_field(name, host_out, capacity);
        if (n == -2) return fail(std::string("evp_get_field: unknown field ") + name, -7);
        if (n < 0) return fail("evp_get_field: buffer too small", -7);
        if (written) *written = n;
    } catch (SolveError& e) {
        return fail(e.what(), e.code);
    }
    return 0;
}

int evp_last_rows(evp_solve* h, double* r51, double* d44) {
    if (!h) return fail("evp_last_rows: null handle", -7);
    if (r51) std::memcpy(r51, h->s.last_results, sizeof(h->s.last_results));
    if (d44) std::memcpy(d44, h->s.last_diag, sizeof(h->s.last_diag));
    return 0;
}

int evp_stats(evp_solve* h, evp_report* r) {
    if (!h || !r) return fail("evp_stats: null argument", -7);
    r->status = 0;
    r->macrosteps = h->s.macrosteps_done;
    r->equilibrium_iters = h->s.total_iters;
    r->voxel_iters = h->s.total_iters * h->s.d.N;
    r->wall_s = 0.0;
    r->gpu_s = h->s.gpu_ms * 1e-3;
    r->n1 = h->s.d.n1; r->n2 = h->s.d.n2; r->n3 = h->s.d.n3;
    r->h2d_bytes = h->s.h2d;
    r->d2h_bytes = h->s.d2h;
    return 0;
}

int evp_kernel_times(evp_solve* h, char* names, long long* launches, double* ms, int cap) {
    if (!h) return fail("evp_kernel_times: null handle", -7);
    const auto& kt = h->s.ktimes;
    int n = 0;
    for (const auto& k : kt) {
        if (n >= cap) break;
        if (names) {
            std::strncpy(names + 32 * n, k.name.c_str(), 31);
            names[32 * n + 31] = '\0';
        }
        if (launches) launches[n] = k.n;
        if (ms) ms[n] = k.ms;
        n++;
    }
    return n;
}

int evp_set_deadline(evp_solve* h, double seconds) {
    if (!h) return fail("evp_set_deadline: null handle", -7);
    h->s.has_deadline = seconds > 0.0;
    h->s.deadline = std::chrono::steady_clock::now() +
                    std::chrono::duration_cast<std::chrono::steady_clock::duration>(std::chrono::duration<double>(seconds > 0.0 ? seconds : 0.0));
    return 0;
}

long long evp_kernel_launches(evp_solve* h) { return h ? h->s.launches : -1; }

int evp_newton_stats(evp_solve* h, long long* out6) {
    if (!h || !out6) return fail("evp_newton_stats: null argument", -7);
    if (!h->s.d.nstats) return fail("evp_newton_stats: the solve was not opened with EVP_PROFILE", -7);
    unsigned long long v[8];
    try {
        CK(cudaMemcpyAsync(v, h->s.d.nstats, sizeof(v), cudaMemcpyDeviceToHost, h->s.st));
        h->s.sync();
    } catch (SolveError& e) {
        return fail(e.what(), e.code);
    }
    for (int i = 0; i < 6; i++) out6[i] = (long long)v[i];
    return 0;
}

int evp_close(evp_solve* h) {
    delete h;
    return 0;
}

struct evp_batch {
    evp::Batch* b = nullptr;
};

int evp_batch_open(evp_batch** out) {
    if (!out) return fail("evp_batch_open: null argument", -7);
    *out = nullptr;
    int dev_count = 0;
    if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0) return fail("no CUDA device available", -6);
    try {
        evp_batch* h = new evp_batch();
        h->b = evp::batch_create(0);
        *out = h;
    } catch (SolveError& e) {
        return fail(e.what(), e.code);
    }
    return 0;
}

int evp_batch_add(evp_batch* h, const char* fft_in, const char* out_dir, int mix, int modal, int flags, int* slot) {
    if (!h || !fft_in || !slot) return fail("evp_batch_add: null argument", -7);
    evp::Deck dk;
    try {
        dk = evp::parse_deck(fft_in);
    } catch (evp::DeckError& e) {
        return fail(e.what(), e.code);
    } catch (std::exception& e) {
        return fail(e.what(), -1);
    }
    std::string err;
    try {
        *slot = evp::batch_add(h->b, std::move(dk), fft_in, out_dir ? out_dir : "", mix, modal, flags, 0.0, err);
    } catch (SolveError& e) {
        return fail(e.what(), e.code);
    }
    int status = 0;
    evp::batch_slot(h->b, *slot, &status, nullptr, nullptr);
    if (status != 0) return fail(err, status);
    return 0;
}

int evp_batch_step(evp_batch* h, int rounds, int* running) {
    if (!h) return fail("evp_batch_step: null handle", -7);
    try {
        const int n = evp::batch_step(h->b, rounds > 0 ? rounds : 1);
        if (running) *running = n;
    } catch (SolveError& e) {
        return fail(e.what(), e.code);
    } catch (std::exception& e) {
        return fail(e.what(), -1);
    }
    return 0;
}

int evp_batch_status(evp_batch* h, int slot, int* state, evp_report* rep, char* msg, int msgcap) {
    if (!h) return fail("evp_batch_status: null handle", -7);
    int status = 0;
    std::string err;
    const int s = evp::batch_slot(h->b, slot, &status, rep, &err);
    if (s < 0) return fail("evp_batch_status: no such slot", -7);
    if (state) *state = s;
    if (msg && msgcap > 0) {
        std::strncpy(msg, err.c_str(), (size_t)msgcap - 1);
        msg[msgcap - 1] = '\0';
    }
    return 0;
}

int evp_batch_close(evp_batch* h) {
    if (!h) return 0;
    evp::batch_destroy(h->b);
    delete h;
    return 0;
}

int evp_solve_files(int n, const char* const* fft_in, const char* const* out_dir, int mix, int modal, int flags,
                    evp_report* reports) {
    if (n < 0 || (n > 0 && (!fft_in || !reports))) return fail("evp_solve_files: null argument", -7);
    evp_batch* h = nullptr;
    int rc = evp_batch_open(&h);
    if (rc != 0) return rc;
    std::vector<int> slots(n, -1);
    int worst = 0;
    for (int i = 0; i < n; i++) {
        const int r = evp_batch_add(h, fft_in[i], out_dir ? out_dir[i] : "", mix, modal,
                                    flags ? flags : EVP_WRITE_FILES, &slots[i]);
        if (r != 0 && slots[i] < 0) {
            std::memset(&reports[i], 0, sizeof(evp_report));
            reports[i].status = r;
            worst = worst ? worst : r;
        }
    }
    int running = 1;
    while (running > 0) {
        rc = evp_batch_step(h, 16, &running);
        if (rc != 0) {
            evp_batch_close(h);
            return rc;
        }
    }
    for (int i = 0; i < n; i++) {
        if (slots[i] < 0) continue;
        int state = 0;
        evp_batch_status(h, slots[i], &state, &reports[i], nullptr, 0);
        if (reports[i].status != 0 && worst == 0) worst = reports[i].status;
    }
    evp_batch_close(h);
    return worst;
}

int evp_tune_cache(const char* path) {
    try {
        const std::string p = path ? path : "";
        if (!p.empty()) {
            const std::string dir = std::filesystem::path(p).parent_path().string();
            if (!dir.empty()) evp::mkdir_p(dir);
        }
        evp::fft_tune_cache(p);
    } catch (std::exception& e) {
        return fail(e.what(), -7);
    }
    return 0;
}

int evp_solve_file(const char* fft_in, const char* out_dir, int nthreads, const char* fftw_save, int mix, int modal, evp_report* report) {
    (void)nthreads;
    if (fftw_save && fftw_save[0]) evp_tune_cache(fftw_save);
    auto t0 = std::chrono::steady_clock::now();
    evp_solve* h = nullptr;
    // the files are only needed when the solve returns: VTK files are written in the background
    int rc = open_solve(fft_in, out_dir, mix, modal, EVP_WRITE_FILES, true, &h);
    if (rc != 0) {
        if (report) { std::memset(report, 0, sizeof(*report)); report->status = rc; }
        return rc;
    }
    int done = 0;
    while (true) {
        rc = evp_advance(h, 1, &done);
        if (rc != 0 || done == 0) break;
    }
    try {
        h->s.wait_vtk();
    } catch (SolveError& e) {
        if (rc == 0) rc = fail(e.what(), e.code);
    } catch (std::exception& e) {
        if (rc == 0) rc = fail(e.what(), -1);
    }
    if (report) {
        evp_stats(h, report);
        report->status = rc;
        report->wall_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    evp_close(h);
    return rc;
}

}  // extern "C"
