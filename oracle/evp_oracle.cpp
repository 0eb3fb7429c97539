// evp_oracle.cpp -- CPU FP64 oracle of the LS-EVPFFT solve.
//
// TEST INFRASTRUCTURE ONLY.  This file restates, routine by routine, the
// reference Fortran solver of gdebrun2/creep_modeling:
//   lsevpfft/src/LS-EVPFFT.f90      driver (cited per block below)
//   lsevpfft/src/various_functions.f90, types.f90, IO_functions.f90,
//   tensor_functions.f90, fourier_functions.f90
// It keeps the reference's array-of-structs voxel record and its loop order;
// reductions run serially in voxel order (the reference's 1-thread order), so
// results do not depend on the thread count.  Built without -ffast-math and
// with -ffp-contract=off (strict IEEE FP64).
//
// Parity status: UNPINNED against the Fortran executable (no Fortran
// toolchain, FFTW or LAPACK in this environment; the reference ships no
// outputs).  Pinned by analytic known-answer tests and numpy/scipy golden
// vectors under tests/golden/.
//
// Deliberate, documented differences from the reference:
//   * grain ids above ngrmx=1000 are accepted (IO_functions.f90:122-125 stops);
//   * IWSTEP=0 means "never write VTK" (LS-EVPFFT.f90:527 divides by zero);
//   * cell2node uses npts1 for the x wrap (various_functions.f90:2678 uses
//     npts2; identical for the cubic grids the decks use).
#include "evp_oracle.h"
#include "or_math.hpp"
#include "or_deck.hpp"

#include <cstdio>
#include <ctime>
#include <string>
#include <vector>
#include <sys/stat.h>
#include <unistd.h>
#ifdef _OPENMP
#include <omp.h>
#endif

using namespace orc;

namespace {

const int NSYSMX = 24;  // global.f90:16
const int NMODMX = 3;   // global.f90:15

struct SolveError : std::runtime_error {
    int code;
    SolveError(const std::string& m, int c) : std::runtime_error(m), code(c) {}
};

// phase_type (types.f90:96-118)
struct Phase {
    bool igas = false;
    int nsyst = 0, nmodes = 0, nsm[NMODMX] = {0, 0, 0};
    double dnca[NSYSMX][3] = {}, dbca[NSYSMX][3] = {}, schca[NSYSMX][5] = {};
    double tau[NSYSMX][3] = {}, hard[NSYSMX][NSYSMX] = {}, thet[NSYSMX][2] = {};
    double nrs[NSYSMX] = {}, gamd0[NSYSMX] = {}, twsh[NSYSMX] = {}, hpfac[NSYSMX] = {};
    T4 C = {};
};

// process_type (types.f90:120-152)
struct Process {
    int ithermo = 0, iudot[3][3] = {}, idsim[6] = {}, iscau[6] = {}, ictrl = 0, nsteps = 0, itmax = 0;
    int irecover = 0, isave = 0, iupdate = 0, iuphard = 0, iwtex = 0, iwfields = 0, iwstep = 0, igamma = 0;
    M3 udot = {}, dsim = {}, tomtot = {}, scauchy = {}, dsim_snapshot = {}, scauchy_snapshot = {};
    double dvm = 0, tdot = 0, tdotref = 0, tdotmin = 0, devmmx = 0, error = 0, erroral = 0, xc0 = 0, devmapp = 0;
};

// voxel_type (types.f90:5-53), trimmed to the fields the solve reads.
struct Voxel {
    double wgtc;
    M3 sg, velgrad;
    int grain, phase;
    bool gas;
    M6 cg66, sg66;
    M3 ag;
    double gacumgr;
    double crss[NSYSMX][2], trialtau[NSYSMX][2];
    M3 eth, F, Fe, Fp, Finv, edotp;
    double epvm;
    M3 sgt, disgradsym;
    double detF;
    M3 Fini;
    double gamdot[NSYSMX], sch[NSYSMX][5];
    M6 c066mod, cG, cgas;
    M3 sgPK1, dvelgradref, velgradold, ept, Finc, Feinc;
    M3 s_velgrad, s_velgradold, s_sg, s_edotp;
    double s_gamdot[NSYSMX], s_trialtau[NSYSMX][2];
};

// diag_type (types.f90:174-249)
struct Diag {
    double detF_min = 0, detF_min_sol = 0, detF_min_gas = 0;
    double detF_min_prev = 0, detF_min_ratio = 1, detF_min_relstep = 0;
    double detF_min_sol_prev = 0, detF_min_sol_ratio = 1, detF_min_sol_relstep = 0;
    double detF_min_gas_prev = 0, detF_min_gas_ratio = 1, detF_min_gas_relstep = 0;
    double volinc_max_sol = 0, volinc_max_gas = 0, volinc_max_sol_prev = 0, volinc_max_gas_prev = 0;
    double volinc_max_sol_relstep = 0, volinc_max_gas_relstep = 0;
    double stretchinc_max_sol = 0, stretchinc_max_gas = 0, stretchinc_max_sol_prev = 0, stretchinc_max_gas_prev = 0;
    double stretchinc_max_sol_relstep = 0, stretchinc_max_gas_relstep = 0;
    double rotang_max_sol = 0, rotang_max_gas = 0, rotang_max_sol_prev = 0, rotang_max_gas_prev = 0;
    double dL_step_rms_sol = 0, dL_step_rms_gas = 0, dL_step_rms = 0, dL_step_max_sol = 0, dL_step_max_gas = 0, dL_step_max = 0;
    double dvelgradavg_mag = 0, erre = 0, errs = 0, errsbc = 0, tdotref = 0, devm_inc_max = 0;
    double s33_target = 0, s33 = 0, s33_sol = 0;
    double cond_c066mod_max_sol = 0, cond_c066mod_max_gas = 0, cond_cgas_max = 0;
    int imin_sol[3] = {0, 0, 0}, imin_gas[3] = {0, 0, 0};
};

inline double safe_rel_change(double x, double xp) {
    if (xp <= TINY || xp >= HUGE_ * 0.5) return 0.0;
    return std::fabs(x - xp) / xp;
}
inline double safe_ratio(double x, double xp) {
    if (xp <= TINY || xp >= HUGE_ * 0.5) return 1.0;
    return x / xp;
}
inline double clamp_subnormal(double a) { return (std::fabs(a) < TINY) ? 0.0 : a; }

// rotate a 4th-order tensor: out_ijkl = sum A_iI A_jJ A_kK A_lL in_IJKL
void rotate4(const M3 A, const T4 in, T4 out) {
    T4 t1, t2;
    for (int i = 0; i < 3; i++) for (int J = 0; J < 3; J++) for (int K = 0; K < 3; K++) for (int L = 0; L < 3; L++) {
        double s = 0; for (int I = 0; I < 3; I++) s += A[i][I] * in[I][J][K][L]; t1[i][J][K][L] = s; }
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) for (int K = 0; K < 3; K++) for (int L = 0; L < 3; L++) {
        double s = 0; for (int J = 0; J < 3; J++) s += A[j][J] * t1[i][J][K][L]; t2[i][j][K][L] = s; }
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) for (int k = 0; k < 3; k++) for (int L = 0; L < 3; L++) {
        double s = 0; for (int K = 0; K < 3; K++) s += A[k][K] * t2[i][j][K][L]; t1[i][j][k][L] = s; }
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) for (int k = 0; k < 3; k++) for (int l = 0; l < 3; l++) {
        double s = 0; for (int L = 0; L < 3; L++) s += A[l][L] * t1[i][j][k][L]; out[i][j][k][l] = s; }
}

std::string fmt_g0(double x) {
    char b[64];
    std::snprintf(b, sizeof(b), "%.17g", x);
    return b;
}
// Fortran Ew.dEe editing used by write_vtk_cell: E18.8E3
std::string fmt_e18_8e3(double x) {
    char m[64], out[64];
    if (x == 0.0) {
        std::snprintf(out, sizeof(out), "%18s", "0.00000000E+000");
        return out;
    }
    std::snprintf(m, sizeof(m), "%.7e", std::fabs(x));  // d.dddddddde+XX
    int e10 = std::atoi(m + 10) + 1;
    char digits[9];
    digits[0] = m[0];
    std::memcpy(digits + 1, m + 2, 7);
    digits[8] = '\0';
    char body[40];
    std::snprintf(body, sizeof(body), "%s0.%sE%c%03d", x < 0 ? "-" : "", digits, e10 < 0 ? '-' : '+', std::abs(e10));
    std::snprintf(out, sizeof(out), "%18s", body);
    return out;
}

void mkdir_p(const std::string& d) {
    std::string cur;
    for (size_t i = 0; i <= d.size(); i++) {
        if (i == d.size() || d[i] == '/') {
            if (!cur.empty()) ::mkdir(cur.c_str(), 0755);
        }
        if (i < d.size()) cur += d[i];
    }
}

struct Oracle {
    // ---- props_type
    int n1 = 0, n2 = 0, n3 = 0, n3node = 1;
    long N = 0;
    int nph = 0, imicrosave = 0, nproc = 0, idispini = 0;
    double wgt = 0, complgas = 0, wphsol = 0, wphgas = 0;
    bool modAL = true;
    std::vector<Phase> phase;
    std::vector<Process> process;
    // ---- micro_type
    M6 c066 = {}, s066 = {};
    T4 c0 = {}, s0 = {}, Goperr0 = {}, de_ds = {};
    double wphcsol = 0, wphcgas = 0;
    M3 defgradavg, defgradinvavgc, defgradinvavgcs, defgradinvavgcg;
    M3 dvelgradavg = {}, velgradavg = {}, velgradavgsol = {}, velgradavggas = {};
    M3 sgavg = {}, sgavgsol = {}, sgsolavg = {};
    double svmavg = 0, dvmavg = 0, edotvmmx = 0, evmavg = 0;
    M3 epavg = {}, eavg = {}, eelavg = {}, edotpavg = {};
    double evmpavg = 0, dvmpavg = 0, lvmavg = 0;
    std::vector<double> Goper;  // 81 per frequency
    std::vector<double> xnode;  // 3 per node
    std::vector<Voxel> vox;
    Diag diag;
    // ---- driver state (global.f90:19-27 and LS-EVPFFT.f90:15-82)
    int ipr = 0, imacroloop = 1, imicro = 0, iter = 0;
    double erre = 0, errs = 0, errsbc = 0;
    double mix = 1.0, sim_time = 0.0, wall_time = 0.0, tdot_plan = 0, proc_time_target = 0, proc_time_done = 0;
    int nconverged = 0, total_macrosteps = 0;
    bool kinematic_controlled = false, do_mix = true;
    long total_iters = 0;
    time_t start = 0;
    bool finished = false;
    // ---- FFT
    Fft1 pf[3], pb[3];
    std::vector<cplx> grid;
    // ---- outputs
    std::string outdir;
    bool write_files = false, verbose = false;
    double last_results[51] = {}, last_diag[44] = {};

    long vidx(int i, int j, int k) const { return i + (long)n1 * (j + (long)n2 * k); }
    Process& P() { return process[ipr - 1]; }

    // ------------------------------------------------------------ init_micro (types.f90:256-343)
    void init_micro() {
        n3node = (n3 == 1) ? 1 : n3 + 1;
        N = (long)n1 * n2 * n3;
        xnode.assign(3L * (n1 + 1) * (n2 + 1) * n3node, 0.0);
        for (int k = 0; k < n3node; k++)
            for (int j = 0; j < n2 + 1; j++)
                for (int i = 0; i < n1 + 1; i++) {
                    long p = 3L * (i + (long)(n1 + 1) * (j + (long)(n2 + 1) * k));
                    xnode[p + 0] = (double)(i + 1) - 0.5;
                    xnode[p + 1] = (double)(j + 1) - 0.5;
                    xnode[p + 2] = (n3node == 1) ? 0.0 : (double)(k + 1) - 0.5;
                }
        vox.assign(N, Voxel());
        for (long v = 0; v < N; v++) {
            Voxel& x = vox[v];
            std::memset(&x, 0, sizeof(Voxel));
            x.wgtc = wgt;
            eye3(x.F); eye3(x.Fe); eye3(x.Fp); eye3(x.Finv); eye3(x.Fini); eye3(x.Finc); eye3(x.Feinc);
            x.detF = 1.0;
        }
        eye3(defgradavg); eye3(defgradinvavgc); eye3(defgradinvavgcs); eye3(defgradinvavgcg);
        for (int a = 0; a < 3; a++) {
            int n = (a == 0) ? n1 : (a == 1) ? n2 : n3;
            pf[a].init(n, -1);
            pb[a].init(n, +1);
        }
        grid.assign(9 * N, cplx(0, 0));
        Goper.assign(81 * N, 0.0);
    }

    // ------------------------------------------------------------ data_crystal (IO_functions.f90:367-638)
    void data_crystal(const std::string& path, int iph) {
        RecordReader r(path);
        Phase& ph = phase[iph];
        r.read_line();
        std::string icryst = r.read_line().substr(0, 3);
        std::vector<double> cdim = r.read_reals(3);
        double covera = cdim[2] / cdim[0];
        int nmodesx = (int)r.read_ints(1)[0];
        int nmodes = (int)r.read_ints(1)[0];
        std::vector<long> mode = r.read_ints(nmodes);
        ph.nmodes = nmodes;
        if (nmodes > NMODMX) throw DeckError("nmodes in phase exceeds nmodmx");
        if (nmodesx > 10) throw DeckError("nmodesx exceeds 10");
        double hselfx[10] = {}, hlatex[10][10] = {};
        int ntwmod = 0, nsyst = 0, kount = 1;
        bool hex = (icryst == "HEX" || icryst == "TRI" || icryst == "hex" || icryst == "tri");
        bool cub = (icryst == "CUB" || icryst == "ORT" || icryst == "cub" || icryst == "ort");
        for (int nm = 1; nm <= nmodesx; nm++) {
            r.read_line();
            std::vector<std::string> t = r.read_tokens(6);
            if (t.size() < 6) throw DeckError("bad mode line in " + path);
            int modex = (int)r.to_int(t[0]), nsmx = (int)r.to_int(t[1]);
            double nrsx = r.to_real(t[2]), gamd0x = r.to_real(t[3]), twshx = r.to_real(t[4]);
            int isectwx = (int)r.to_int(t[5]);
            (void)isectwx;
            std::vector<double> h = r.read_reals(6);
            double tau0xf = h[0], tau0xb = h[1], tau1x = h[2], thet0x = h[3], thet1x = h[4], hpfacx = h[5];
            std::vector<double> hl = r.read_reals(1 + nmodesx);
            hselfx[nm - 1] = hl[0];
            for (int jm = 0; jm < nmodesx; jm++) hlatex[nm - 1][jm] = hl[1 + jm];
            if (kount > nmodes || modex != mode[kount - 1]) {
                for (int iz = 0; iz < nsmx; iz++) r.skip();
                continue;
            }
            if (thet0x < thet1x) throw DeckError("initial hardening lower than final hardening");
            if (tau1x <= 1.e-6) { tau1x = 1.e-6; thet0x = thet1x; }
            hselfx[kount - 1] = hselfx[nm - 1];
            for (int i = 0; i < nmodes; i++) hlatex[kount - 1][i] = hlatex[nm - 1][mode[i] - 1];
            std::vector<std::vector<long>> isn(nsmx), isb(nsmx);
            if (hex) {
                for (int j = 0; j < nsmx; j++) { auto v = r.read_ints(8); isn[j] = {v[0], v[1], v[2], v[3]}; isb[j] = {v[4], v[5], v[6], v[7]}; }
            } else if (cub) {
                for (int j = 0; j < nsmx; j++) { auto v = r.read_ints(6); isn[j] = {v[0], v[1], v[2]}; isb[j] = {v[3], v[4], v[5]}; }
            } else {
                throw DeckError("cannot identify the crystal symmetry");
            }
            ph.nsm[kount - 1] = nsmx;
            if (twshx > 1.0e-15) ntwmod++;
            if (ntwmod > 0) throw DeckError("twinning modes are not supported (ntwmmx = 0)");
            for (int js = 0; js < nsmx; js++) {
                nsyst++;
                if (nsyst > NSYSMX) throw DeckError("nsyst exceeds nsysmx");
                int s = nsyst - 1;
                ph.gamd0[s] = gamd0x; ph.nrs[s] = nrsx; ph.twsh[s] = twshx;
                ph.tau[s][0] = tau0xf; ph.tau[s][1] = tau0xb; ph.tau[s][2] = tau1x;
                ph.thet[s][0] = thet0x; ph.thet[s][1] = thet1x; ph.hpfac[s] = hpfacx;
                double sn[3], sb[3];
                if (hex) {
                    sn[0] = (double)isn[js][0];
                    sn[1] = ((double)isn[js][0] + 2. * (double)isn[js][1]) / std::sqrt(3.);
                    sn[2] = (double)isn[js][3] / covera;
                    sb[0] = 3. / 2. * (double)isb[js][0];
                    sb[1] = ((double)isb[js][0] / 2. + (double)isb[js][1]) * std::sqrt(3.);
                    sb[2] = (double)isb[js][3] * covera;
                } else {
                    for (int m = 0; m < 3; m++) { sn[m] = (double)isn[js][m] / cdim[m]; sb[m] = (double)isb[js][m] * cdim[m]; }
                }
                double snor = std::sqrt(sn[0] * sn[0] + sn[1] * sn[1] + sn[2] * sn[2]);
                double qnor = std::sqrt(sb[0] * sb[0] + sb[1] * sb[1] + sb[2] * sb[2]);
                double prod = 0.;
                for (int j = 0; j < 3; j++) {
                    ph.dnca[s][j] = sn[j] / snor;
                    ph.dbca[s][j] = sb[j] / qnor;
                    if (std::fabs(ph.dnca[s][j]) < 1.e-03) ph.dnca[s][j] = 0.;
                    if (std::fabs(ph.dbca[s][j]) < 1.e-03) ph.dbca[s][j] = 0.;
                    prod += ph.dnca[s][j] * ph.dbca[s][j];
                }
                if (prod >= 1.e-3) throw DeckError("slip system is not orthogonal");
                M3 a;
                for (int i = 0; i < 3; i++)
                    for (int j = 0; j < 3; j++) a[i][j] = (ph.dnca[s][i] * ph.dbca[s][j] + ph.dnca[s][j] * ph.dbca[s][i]) / 2.;
                t2_to_b5(a, ph.schca[s]);
            }
            ph.nsyst = nsyst;
            kount++;
        }
        int i = 0;
        for (int im = 0; im < nmodes; im++)
            for (int is = 0; is < ph.nsm[im]; is++) {
                int j = 0;
                for (int jm = 0; jm < nmodes; jm++)
                    for (int js = 0; js < ph.nsm[jm]; js++) { ph.hard[i][j] = hlatex[im][jm]; j++; }
                ph.hard[i][i] = hselfx[im];
                i++;
            }
    }

    // ------------------------------------------------------------ data_crystal_elast (IO_functions.f90:640-720)
    void data_crystal_elast(const std::string& path, int iph) {
        RecordReader r(path);
        Phase& ph = phase[iph];
        int iso = (int)r.read_ints(1)[0];
        if (iso == 0) {
            M6 cc;
            for (int i = 0; i < 6; i++) { auto v = r.read_reals(6); for (int j = 0; j < 6; j++) cc[i][j] = v[j]; }
            v66_to_t4(cc, ph.C);
        } else {
            auto v = r.read_reals(2);
            double young = v[0], tnu = v[1];
            double tmu = young / (2.0 * (1. + tnu));
            double tla = 2.0 * tmu * tnu / (1.0 - 2.0 * tnu);
            for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) for (int k = 0; k < 3; k++) for (int l = 0; l < 3; l++) {
                double dij = i == j, dkl = k == l, dik = i == k, djl = j == l, dil = i == l, djk = j == k;
                ph.C[i][j][k][l] = tla * dij * dkl + 2.0 * tmu * ((dik * djl + dil * djk) / 2.0);
            }
        }
    }

    // ------------------------------------------------------------ data_grain (IO_functions.f90:722-812)
    void data_grain(const std::string& path) {
        RecordReader r(path);
        for (long kkk = 0; kkk < N; kkk++) {
            auto t = r.read_tokens(8);
            if (t.size() < 8) throw DeckError("short microstructure record");
            double ph = r.to_real(t[0]), th = r.to_real(t[1]), om = r.to_real(t[2]);
            long ii = r.to_int(t[3]), jj = r.to_int(t[4]), kk = r.to_int(t[5]), jgr = r.to_int(t[6]), jph = r.to_int(t[7]);
            if (ii < 1 || ii > n1 || jj < 1 || jj > n2 || kk < 1 || kk > n3) throw DeckError("voxel index out of range");
            if (jph < 1 || jph > nph) throw DeckError("phase id out of range");
            Voxel& x = vox[vidx(ii - 1, jj - 1, kk - 1)];
            x.grain = (int)jgr;
            x.phase = (int)jph;
            x.gas = phase[jph - 1].igas;
            if (x.gas) continue;
            M3 aa;
            euler2(ph * PI / 180.0, th * PI / 180.0, om * PI / 180.0, aa);
            for (int j = 0; j < 3; j++) for (int k = 0; k < 3; k++) x.ag[j][k] = aa[k][j];
            T4 caux;
            rotate4(x.ag, phase[jph - 1].C, caux);
            t4_to_b66(caux, x.cg66);
            if (inv6(x.cg66, x.sg66) != 0) throw SolveError("Singular matrix in lu_inverse (data_grain)", -3);
        }
    }

    // ------------------------------------------------------------ load_input (IO_functions.f90:6-365)
    void load_input(const std::string& fft_in) {
        RecordReader r(fft_in);
        nph = (int)r.read_ints(1)[0];
        auto g = r.read_ints(3);
        n1 = (int)g[0]; n2 = (int)g[1]; n3 = (int)g[2];
        if (n1 < 1 || n2 < 1 || n3 < 1) throw DeckError("bad grid size");
        if (nph < 1) throw DeckError("bad number of phases");
        wgt = 1.0 / (double)((long)n1 * n2 * n3);
        init_micro();
        r.read_reals(3);  // delt is read and then forced to 4 (IO_functions.f90:62-66)
        double delt[3] = {4, 4, 4};
        r.read_line();
        std::string filetext = trim(r.read_line());
        phase.assign(nph, Phase());
        for (int iph = 0; iph < nph; iph++) {
            r.read_line();
            long ii = r.read_ints(1)[0];
            phase[iph].igas = (ii != 0);
            r.read_line();
            std::string fpl = trim(r.read_line());
            std::string fel = trim(r.read_line());
            if (!phase[iph].igas) {
                data_crystal(fpl, iph);
                data_crystal_elast(fel, iph);
            }
        }
        data_grain(filetext);
        // Hall-Petch startup shift (IO_functions.f90:107-199)
        double hp_kgr_default = 632 / 2.5;
        double voxel_vol = delt[0] * delt[1] * delt[2];
        double grain_dmin = 3.0 * std::pow(voxel_vol, 1.0 / 3.0);
        std::vector<std::vector<long>> grain_nvox(nph);
        for (long v = 0; v < N; v++) {
            const Voxel& x = vox[v];
            if (x.gas) continue;
            if (x.grain < 1) throw DeckError("grain id out of bounds for Hall-Petch init");
            auto& gv = grain_nvox[x.phase - 1];
            if ((long)gv.size() < x.grain + 1) gv.resize(x.grain + 1, 0);
            gv[x.grain]++;
        }
        r.read_line();
        auto rs = r.read_ints(2);
        imicrosave = (int)rs[1];
        complgas = r.read_reals(1)[0];
        r.read_line();
        idispini = (int)r.read_ints(1)[0];
        std::string filedispl;
        if (idispini > 0) {
            if (idispini > 2) throw DeckError("idispini must be 0, 1 or 2");
            filedispl = trim(r.read_line());
            init_defgrad(filedispl);
        }
        for (long v = 0; v < N; v++) {
            Voxel& x = vox[v];
            x.gacumgr = 0.0;
            if (x.gas) continue;
            const Phase& ph = phase[x.phase - 1];
            double hp_shift = 0.0;
            if (hp_kgr_default > 0.0) {
                long nv = grain_nvox[x.phase - 1][x.grain];
                double grain_d = nv > 0 ? std::pow((double)nv * voxel_vol, 1.0 / 3.0) : 0.0;
                if (grain_d > 0.0) {
                    grain_d = std::max(grain_d, grain_dmin);
                    hp_shift = hp_kgr_default / std::sqrt(grain_d);
                }
            }
            for (int i = 0; i < ph.nsyst; i++) {
                x.crss[i][0] = ph.tau[i][0] + hp_shift;
                x.crss[i][1] = ph.tau[i][1] + hp_shift;
                double dbsa[3];
                for (int i1 = 0; i1 < 3; i1++) {
                    double dum = 0.0;
                    for (int j1 = 0; j1 < 3; j1++) dum += x.ag[i1][j1] * ph.dbca[i][j1];
                    dbsa[i1] = dum;
                }
                double cosalpha = std::fabs(dbsa[1]);
                x.crss[i][0] = x.crss[i][0] + ph.hpfac[i] * std::sqrt(cosalpha);
                x.crss[i][1] = x.crss[i][1] + ph.hpfac[i] * std::sqrt(cosalpha);
                x.trialtau[i][0] = x.crss[i][1];  // H2: both columns from the backward CRSS
                x.trialtau[i][1] = x.crss[i][1];
            }
        }
        nproc = (int)r.read_ints(1)[0];
        if (nproc < 1) throw DeckError("cannot have less than one processes");
        process.assign(nproc, Process());
        struct M3w { M3 m; };
        std::vector<M3w> eth_tab;
        for (int p = 0; p < nproc; p++) {
            Process& pr = process[p];
            r.read_line(); r.read_line();
            for (int i = 0; i < 3; i++) { auto v = r.read_ints(3); for (int j = 0; j < 3; j++) pr.iudot[i][j] = (int)v[j]; }
            if (pr.iudot[0][0] + pr.iudot[1][1] + pr.iudot[2][2] == 2) throw DeckError("check diagonal boundary conditions iudot");
            for (int i = 0; i < 3; i++)
                for (int j = 0; j < 3; j++)
                    if (i != j && pr.iudot[i][j] + pr.iudot[j][i] == 0) throw DeckError("check off-diagonal boundary conditions iudot");
            r.skip();
            for (int i = 0; i < 3; i++) { auto v = r.read_reals(3); for (int j = 0; j < 3; j++) pr.udot[i][j] = v[j]; }
            sym33(pr.udot, pr.dsim);
            antisym33(pr.udot, pr.tomtot);
            double dvm = vm_strain(pr.dsim);
            for (int i = 0; i < 3; i++) pr.idsim[i] = pr.iudot[i][i];
            pr.idsim[3] = (pr.iudot[1][2] == 1 && pr.iudot[2][1] == 1) ? 1 : 0;
            pr.idsim[4] = (pr.iudot[0][2] == 1 && pr.iudot[2][0] == 1) ? 1 : 0;
            pr.idsim[5] = (pr.iudot[0][1] == 1 && pr.iudot[1][0] == 1) ? 1 : 0;
            r.skip();
            { auto v = r.read_ints(3); pr.iscau[0] = (int)v[0]; pr.iscau[5] = (int)v[1]; pr.iscau[4] = (int)v[2]; }
            { auto v = r.read_ints(2); pr.iscau[1] = (int)v[0]; pr.iscau[3] = (int)v[1]; }
            { auto v = r.read_ints(1); pr.iscau[2] = (int)v[0]; }
            for (int i = 0; i < 6; i++)
                if (pr.iscau[i] * pr.idsim[i] != 0 || pr.iscau[i] + pr.idsim[i] != 1)
                    throw DeckError("check boundary condits on strain-rate and stress");
            r.skip();
            { auto v = r.read_reals(3); pr.scauchy[0][0] = v[0]; pr.scauchy[0][1] = v[1]; pr.scauchy[0][2] = v[2]; }
            { auto v = r.read_reals(2); pr.scauchy[1][1] = v[0]; pr.scauchy[1][2] = v[1]; }
            { auto v = r.read_reals(1); pr.scauchy[2][2] = v[0]; }
            pr.scauchy[2][1] = pr.scauchy[1][2]; pr.scauchy[2][0] = pr.scauchy[0][2]; pr.scauchy[1][0] = pr.scauchy[0][1];
            r.skip();
            { auto v = r.read_reals(4); pr.tdot = v[0]; pr.tdotref = v[1]; pr.tdotmin = v[2]; pr.devmmx = v[3]; }
            pr.ictrl = (int)r.read_ints(1)[0];
            if (pr.ictrl == 0) {
                pr.devmapp = pr.tdot;
                pr.tdot = pr.tdot / dvm;
                pr.tdotref = pr.tdot;
            } else if (pr.ictrl > 0) {
                throw DeckError("ictrl>0 not implemented");
            }
            r.skip();
            pr.nsteps = (int)r.read_ints(1)[0];
            { auto v = r.read_reals(2); pr.error = v[0]; pr.erroral = v[1]; }
            pr.itmax = (int)r.read_ints(1)[0];
            pr.irecover = (int)r.read_ints(1)[0];
            if (pr.irecover == 1 && access("stress.in", R_OK) != 0) throw DeckError("stress.in not found (IRECOVER=1)");
            pr.isave = (int)r.read_ints(1)[0];
            pr.iupdate = (int)r.read_ints(1)[0];
            pr.iuphard = (int)r.read_ints(1)[0];
            pr.iwtex = (int)r.read_ints(1)[0];
            { auto v = r.read_ints(2); pr.iwfields = (int)v[0]; pr.iwstep = (int)v[1]; }
            { auto t = r.read_tokens(2); if (t.size() < 2) throw DeckError("bad XC0, IGAMMA line"); pr.xc0 = r.to_real(t[0]); pr.igamma = (int)r.to_int(t[1]); }
            if (!(pr.nsteps > 0)) throw DeckError("nsteps must be positive");
            if (!(pr.error > 0 || pr.erroral > 0)) throw DeckError("error and erroral tolerances must be positive");
            if (!(pr.itmax > 0)) throw DeckError("itmax must be positive");
            if (!(pr.irecover == 0 || pr.irecover == 1)) throw DeckError("irecover must be 0 or 1");
            if (!(pr.isave == 0 || pr.isave == 1)) throw DeckError("isave must be 0 or 1");
            if (!(pr.iupdate == 0 || pr.iupdate == 1)) throw DeckError("iupdate must be 0 or 1");
            if (!(pr.iuphard == 0 || pr.iuphard == 1)) throw DeckError("iuphard must be 0 or 1");
            if (!(pr.iwtex == 0 || pr.iwtex == 1)) throw DeckError("iwtex must be 0 or 1");
            if (!(pr.iwfields == 0 || pr.iwfields == 1)) throw DeckError("iwfields must be 0 or 1");
            if (!(pr.igamma == 0 || pr.igamma == 1 || pr.igamma == 2)) throw DeckError("igamma must be 0, 1 or 2");
            pr.ithermo = (int)r.read_ints(1)[0];
            if (pr.ithermo == 1) {
                std::string fth = trim(r.read_line());
                RecordReader th(fth);
                long ngr = th.read_ints(1)[0];
                if ((long)eth_tab.size() < ngr + 1) eth_tab.resize(ngr + 1);
                for (long ig = 1; ig <= ngr; ig++) {
                    auto v = th.read_reals(6);
                    M3& e = eth_tab[ig].m;
                    e[0][0] = v[0]; e[1][1] = v[1]; e[2][2] = v[2]; e[1][2] = v[3]; e[2][0] = v[4]; e[0][1] = v[5];
                    e[2][1] = e[1][2]; e[0][2] = e[2][0]; e[1][0] = e[0][1];
                }
            }
            for (long v = 0; v < N; v++) {
                int gid = vox[v].grain;
                if (gid >= 1 && gid < (long)eth_tab.size()) copy3(eth_tab[gid].m, vox[v].eth);
                else std::memset(vox[v].eth, 0, sizeof(M3));
            }
        }
        wphsol = 0.0; wphgas = 0.0;
        for (long v = 0; v < N; v++) {
            if (vox[v].gas) wphgas += wgt;
            if (!vox[v].gas) wphsol += wgt;
        }
        if (idispini == 0) {
            wphcgas = wphgas;
            wphcsol = wphsol;
        }
    }

    // ------------------------------------------------------------ init_defgrad (IO_functions.f90:815-936)
    // Initial displacement field: cell centres (IDISPINI 1, nodes by cell2node_tensor1) or nodes
    // (IDISPINI 2, cells = the lower-corner nodes); F = grad u + diag(delt) with delt = 4 as forced
    // at IO_functions.f90:62-66; gradient_tensor1 (various_functions.f90:56-112) with ideriv 1 or 2.
    void init_defgrad(const std::string& fdisp) {
        const long nn1 = n1 + 1, nn2 = n2 + 1, nn3 = n3 + 1;
        std::vector<double> u(3 * N), un(3 * nn1 * nn2 * nn3, 0.0);
        auto node = [&](long i, long j, long k) { return 3 * (i + nn1 * (j + nn2 * k)); };
        RecordReader f(fdisp);
        int ideriv;
        if (idispini == 1) {
            for (long v = 0; v < N; v++) {
                auto t = f.read_reals(6);
                for (int l = 0; l < 3; l++) u[3 * v + l] = t[3 + l];
            }
            // cell2node_tensor1 (various_functions.f90:2652-2691), x wrapped with n1
            for (long k = 1; k <= n3 + 1; k++) {
                long k1 = k - 1, k2 = k;
                if (k1 == 0) k1 = n3;
                if (k2 == n3 + 1) k2 = 1;
                for (long j = 1; j <= n2 + 1; j++) {
                    long j1 = j - 1, j2 = j;
                    if (j1 == 0) j1 = n2;
                    if (j2 == n2 + 1) j2 = 1;
                    for (long i = 1; i <= n1 + 1; i++) {
                        long i1 = i - 1, i2 = i;
                        if (i1 == 0) i1 = n1;
                        if (i2 == n1 + 1) i2 = 1;
                        auto c = [&](long a, long b, long cc, int l) { return u[3 * vidx(a - 1, b - 1, cc - 1) + l]; };
                        for (int l = 0; l < 3; l++)
                            un[node(i - 1, j - 1, k - 1) + l] = (c(i2, j2, k2, l) + c(i1, j2, k2, l) + c(i2, j1, k2, l) +
                                                                 c(i2, j2, k1, l) + c(i1, j1, k2, l) + c(i1, j2, k1, l) +
                                                                 c(i2, j1, k1, l) + c(i1, j1, k1, l)) * 0.125;
                    }
                }
            }
            ideriv = 1;
        } else {
            for (long k = 0; k < n3node; k++)
                for (long j = 0; j < nn2; j++)
                    for (long i = 0; i < nn1; i++) {
                        auto t = f.read_reals(6);
                        for (int l = 0; l < 3; l++) un[node(i, j, k) + l] = t[3 + l];
                    }
            for (long v = 0; v < N; v++) {
                long i = v % n1, j = (v / n1) % n2, k = v / ((long)n1 * n2);
                for (int l = 0; l < 3; l++) u[3 * v + l] = un[node(i, j, k) + l];
            }
            ideriv = 2;
        }
        // gradient_tensor1: grad(l, m) = d u_l / d x_m = Re ifft(kmod_m * fft(u_l)) / N
        std::vector<cplx> g3(3 * N), g9(9 * N);
        for (long v = 0; v < N; v++)
            for (int l = 0; l < 3; l++) g3[(long)l * N + v] = cplx(u[3 * v + l], 0.0);
        for (int c = 0; c < 3; c++) fft3_field(&g3[(long)c * N], n1, n2, n3, pf[0], pf[1], pf[2]);
        for (long v = 0; v < N; v++) {
            int i = (int)(v % n1) + 1, j = (int)((v / n1) % n2) + 1, k = (int)(v / ((long)n1 * n2)) + 1;
            double xk[3];
            spatial_freq(i, j, k, xk);
            cplx km[3];
            if (ideriv == 2) {
                cplx base = cplx(0.0, 1.0) * 0.25 * (1.0 + std::exp(cplx(0.0, xk[0]))) * (1.0 + std::exp(cplx(0.0, xk[1]))) *
                            (1.0 + std::exp(cplx(0.0, xk[2])));
                for (int l = 0; l < 3; l++) km[l] = std::tan(xk[l] / 2.0) * base;
            } else {
                for (int l = 0; l < 3; l++) km[l] = cplx(0.0, std::sin(xk[l]));
            }
            for (int l = 0; l < 3; l++)
                for (int m = 0; m < 3; m++) g9[(long)(m * 3 + l) * N + v] = g3[(long)l * N + v] * km[m];
            if ((n1 % 2 == 0 && i == n1 / 2 + 1) && (n2 % 2 == 0 && j == n2 / 2 + 1) && ((n3 % 2 == 0 && k == n3 / 2 + 1) && n3 > 1) &&
                ideriv == 2)
                for (int c = 0; c < 9; c++) g9[(long)c * N + v] = 0.0;
        }
        for (int c = 0; c < 9; c++) fft3_field(&g9[(long)c * N], n1, n2, n3, pb[0], pb[1], pb[2]);
        for (long k = 0; k < n3node; k++)
            for (long j = 0; j < nn2; j++)
                for (long i = 0; i < nn1; i++) {
                    long p = 3L * (i + (long)(n1 + 1) * (j + (long)(n2 + 1) * k));
                    for (int l = 0; l < 3; l++) xnode[p + l] = xnode[p + l] + un[node(i, j, k) + l];
                }
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) defgradavg[a][b] = (a == b) ? 4.0 : 0.0;  // diag(delt)
        M3 sc = {}, scs = {}, scg = {};
        double wsol = 0.0, wgas = 0.0, detFavg = 0.0;
        bool failed = false;
        for (long v = 0; v < N; v++) {
            Voxel& x = vox[v];
            for (int l = 0; l < 3; l++)
                for (int m = 0; m < 3; m++) x.F[l][m] = g9[(long)(m * 3 + l) * N + v].real() / (double)N + defgradavg[l][m];
            copy3(x.F, x.Fini);
            x.detF = det33(x.F);
            if (inv3(x.F, x.Finv) != 0) failed = true;
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++) {
                    const double t = x.Finv[a][b] * wgt * x.detF;
                    sc[a][b] = sc[a][b] + t;
                    if (!x.gas) scs[a][b] = scs[a][b] + t;
                    if (x.gas) scg[a][b] = scg[a][b] + t;
                }
            if (!x.gas) wsol = wsol + wgt * x.detF;
            if (x.gas) wgas = wgas + wgt * x.detF;
            x.wgtc = wgt * x.detF;
            detFavg = detFavg + x.detF * wgt;
        }
        if (failed) throw SolveError("Singular matrix in lu_inverse (init_defgrad)", -3);
        wphcsol = wsol / detFavg;
        wphcgas = wgas / detFavg;
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) {
                defgradinvavgc[a][b] = sc[a][b] / detFavg;
                defgradinvavgcs[a][b] = scs[a][b] / detFavg / wphcsol;
                defgradinvavgcg[a][b] = (wphcgas > 0.0) ? scg[a][b] / detFavg / wphcgas : (a == b ? 1.0 : 0.0);
            }
        for (long v = 0; v < N; v++) vox[v].wgtc = vox[v].wgtc / detFavg;
    }

    // ------------------------------------------------------------ initial_guess (various_functions.f90:8-53)
    void initial_guess() {
        const Process& p1 = process[0];
        for (long v = 0; v < N; v++) {
            Voxel& x = vox[v];
            copy3(p1.udot, x.velgrad);
            if (!x.gas) {
                double udot6[6], sg6[6];
                t2_to_b6(p1.udot, udot6);
                for (int i = 0; i < 6; i++) {
                    double s = 0;
                    for (int j = 0; j < 6; j++) s += x.cg66[i][j] * (udot6[j] * p1.tdot);
                    sg6[i] = s;
                }
                b6_to_t2(sg6, x.sg);
            }
        }
        dvmavg = vm_strain(p1.dsim);
        lvmavg = dvmavg;
    }

    // ------------------------------------------------------------ update_schmid (various_functions.f90:472-539)
    void update_schmid() {
        bool failed = false;
#pragma omp parallel for schedule(static)
        for (long v = 0; v < N; v++) {
            Voxel& x = vox[v];
            if (x.gas) continue;
            const Phase& ph = phase[x.phase - 1];
            M3 aa, aainv;
            matmul3(x.Fe, x.ag, aa);
            if (inv3(aa, aainv) != 0) { failed = true; continue; }
            for (int is = 0; is < ph.nsyst; is++) {
                M3 s, t, r, rs;
                for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) s[i][j] = ph.dbca[is][i] * ph.dnca[is][j];
                matmul3(aa, s, t);
                matmul3(t, aainv, r);
                sym33(r, rs);
                t2_to_b5(rs, x.sch[is]);
            }
        }
        if (failed) throw SolveError("Singular matrix in lu_inverse (update_schmid)", -3);
    }

    // ------------------------------------------------------------ spatial_freq (fourier_functions.f90:340-371)
    void spatial_freq(int x, int y, int z, double xi[3]) const {
        const double twopi = 8.0 * std::atan(1.0);
        xi[0] = (x <= n1 / 2) ? twopi * (double)(x - 1) / (double)n1 : twopi * (double)(x - n1 - 1) / (double)n1;
        xi[1] = (y <= n2 / 2) ? twopi * (double)(y - 1) / (double)n2 : twopi * (double)(y - n2 - 1) / (double)n2;
        if (n3 == 1) xi[2] = 0.;
        else xi[2] = (z <= n3 / 2) ? twopi * (double)(z - 1) / (double)n3 : twopi * (double)(z - n3 - 1) / (double)n3;
    }

    // ------------------------------------------------------------ form_G (various_functions.f90:609-809)
    void form_G() {
        const int igamma = P().igamma;
        bool ok = true;
#pragma omp parallel for schedule(static)
        for (long v = 0; v < N; v++) {
            int kxx = (int)(v % n1) + 1, kyy = (int)((v / n1) % n2) + 1, kzz = (int)(v / ((long)n1 * n2)) + 1;
            double xk[3];
            spatial_freq(kxx, kyy, kzz, xk);
            bool nx = (n1 % 2 == 0 && kxx == n1 / 2 + 1), ny = (n2 % 2 == 0 && kyy == n2 / 2 + 1);
            bool nz = (n3 % 2 == 0 && kzz == n3 / 2 + 1);
            T4 g1;
            if ((nx || ny || (nz && n3 > 1)) && igamma == 0) {
                for (int i = 0; i < 81; i++) (&g1[0][0][0][0])[i] = -(&s0[0][0][0][0])[i];
            } else if (((nx && ny) || (nx && nz) || (ny && nz)) && igamma >= 2) {
                std::memset(g1, 0, sizeof(T4));
            } else {
                M3 D;
                if (igamma == 0) {
                    for (int ii = 0; ii < 3; ii++) for (int jj = 0; jj < 3; jj++) D[ii][jj] = xk[ii] * xk[jj];
                } else if (igamma == 1) {
                    double xisum = 2. * PI * (double)(kxx - 1) / (double)n1;
                    double xjsum = 2. * PI * (double)(kyy - 1) / (double)n2;
                    double xksum = 2. * PI * (double)(kzz - 1) / (double)n3;
                    D[0][0] = 2.0 * (std::cos(xisum) - 1.0);
                    D[1][1] = 2.0 * (std::cos(xjsum) - 1.0);
                    D[2][2] = 2.0 * (std::cos(xksum) - 1.0);
                    D[1][0] = -std::sin(xisum) * std::sin(xjsum);
                    D[2][0] = -std::sin(xisum) * std::sin(xksum);
                    D[2][1] = -std::sin(xjsum) * std::sin(xksum);
                    D[0][1] = D[1][0]; D[0][2] = D[2][0]; D[1][2] = D[2][1];
                } else {
                    cplx km[3];
                    cplx base = cplx(0.0, 1.0) * 0.25 * (1.0 + std::exp(cplx(0.0, xk[0]))) * (1.0 + std::exp(cplx(0.0, xk[1]))) *
                                (1.0 + std::exp(cplx(0.0, xk[2])));
                    for (int ii = 0; ii < 3; ii++) km[ii] = std::tan(xk[ii] / 2.0) * base;
                    double im2 = 0.0;
                    for (int ii = 0; ii < 3; ii++)
                        for (int jj = 0; jj < 3; jj++) {
                            cplx d = km[ii] * std::conj(km[jj]);
                            D[ii][jj] = d.real();
                            im2 += d.imag() * d.imag();
                        }
                    if (std::sqrt(im2) > 1.0e-7) ok = false;
                }
                M3 a;
                if (kxx == 1 && kyy == 1 && kzz == 1) {
                    std::memset(a, 0, sizeof(M3));
                } else {
                    for (int i = 0; i < 3; i++)
                        for (int k = 0; k < 3; k++) {
                            double s = 0.;
                            for (int j = 0; j < 3; j++)
                                for (int l = 0; l < 3; l++) s += c0[i][j][k][l] * D[j][l];
                            a[i][k] = s;
                        }
                    M3 ai;
                    if (inv3(a, ai) != 0) ok = false;
                    copy3(ai, a);
                }
                for (int p = 0; p < 3; p++) for (int q = 0; q < 3; q++) for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++)
                    g1[p][q][i][j] = -a[p][i] * D[q][j];
            }
            if (igamma == 1) {
                T4 gt, aux;
                std::memcpy(gt, g1, sizeof(T4));
                for (int itt = 0; itt < 4; itt++) {
                    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) for (int k = 0; k < 3; k++) for (int l = 0; l < 3; l++) {
                        double dum = 0.0;
                        for (int m = 0; m < 3; m++) for (int n = 0; n < 3; n++) for (int o = 0; o < 3; o++) for (int p = 0; p < 3; p++)
                            dum -= g1[i][j][m][n] * c0[m][n][o][p] * gt[o][p][k][l];
                        aux[i][j][k][l] = dum;
                    }
                    std::memcpy(gt, aux, sizeof(T4));
                }
                std::memcpy(g1, gt, sizeof(T4));
            }
            std::memcpy(&Goper[81 * v], g1, sizeof(T4));
        }
        if (!ok) throw SolveError("form_G failed (singular acoustic tensor or complex D operator)", -3);
        // Goperr0 = real part of the inverse DFT at the origin (various_functions.f90:798-807)
        for (int c = 0; c < 81; c++) {
            double s = 0.0;
            for (long v = 0; v < N; v++) s += Goper[81 * v + c];
            (&Goperr0[0][0][0][0])[c] = s / (double)N;
        }
    }

    // ------------------------------------------------------------ calc_c066mod_Goperr066mod (various_functions.f90:812-906)
    void calc_c066mod() {
#pragma omp parallel for schedule(static)
        for (long v = 0; v < N; v++) {
            Voxel& x = vox[v];
            T4 c0mod, c0s;
            for (int ii = 0; ii < 3; ii++) for (int jj = 0; jj < 3; jj++) for (int kk = 0; kk < 3; kk++) for (int ll = 0; ll < 3; ll++) {
                double dum = 0.0;
                for (int m = 0; m < 3; m++) for (int n = 0; n < 3; n++) dum += c0[ii][m][kk][n] * x.F[jj][m] * x.F[ll][n];
                c0mod[ii][jj][kk][ll] = dum / x.detF;
            }
            for (int ii = 0; ii < 3; ii++) for (int jj = 0; jj < 3; jj++) for (int kk = 0; kk < 3; kk++) for (int ll = 0; ll < 3; ll++)
                c0s[ii][jj][kk][ll] = 0.25 * (c0mod[ii][jj][kk][ll] + c0mod[jj][ii][kk][ll] + c0mod[ii][jj][ll][kk] + c0mod[jj][ii][ll][kk]);
            t4_to_b66(c0s, x.c066mod);
            if (modAL) {
                T4 gm, gs;
                M6 g66;
                for (int ii = 0; ii < 3; ii++) for (int jj = 0; jj < 3; jj++) for (int kk = 0; kk < 3; kk++) for (int ll = 0; ll < 3; ll++) {
                    double dum = 0.0;
                    for (int m = 0; m < 3; m++) for (int n = 0; n < 3; n++) dum += Goperr0[ii][m][kk][n] * x.Finv[m][jj] * x.Finv[n][ll];
                    gm[ii][jj][kk][ll] = dum * x.detF;
                }
                for (int ii = 0; ii < 3; ii++) for (int jj = 0; jj < 3; jj++) for (int kk = 0; kk < 3; kk++) for (int ll = 0; ll < 3; ll++)
                    gs[ii][jj][kk][ll] = 0.25 * (gm[ii][jj][kk][ll] + gm[jj][ii][kk][ll] + gm[ii][jj][ll][kk] + gm[jj][ii][ll][kk]);
                t4_to_b66(gs, g66);
                for (int i = 0; i < 6; i++) for (int j = 0; j < 6; j++) {
                    double s = 0; for (int k = 0; k < 6; k++) s += x.c066mod[i][k] * g66[k][j]; x.cG[i][j] = s; }
            }
        }
    }

    // ------------------------------------------------------------ calc_gas_compl (various_functions.f90:909-951)
    void calc_gas_compl() {
        for (long v = 0; v < N; v++) {
            Voxel& x = vox[v];
            if (x.gas) {
                M6 a;
                for (int i = 0; i < 6; i++) for (int j = 0; j < 6; j++) {
                    a[i][j] = (i == j ? 1.0 : 0.0) + x.c066mod[i][j] / P().tdot * complgas;
                    if (modAL) a[i][j] -= x.cG[i][j];
                }
                if (inv6(a, x.cgas) != 0) throw SolveError("Singular matrix in lu_inverse (calc_gas_compl)", -3);
            } else {
                std::memset(x.cgas, 0, sizeof(M6));
            }
        }
    }

    // ------------------------------------------------------------ convolution_with_Goper (various_functions.f90:966-1059)
    void convolution() {
        for (long v = 0; v < N; v++)
            for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) grid[(long)(i * 3 + j) * N + v] = cplx(vox[v].sgPK1[i][j], 0.0);
        for (int c = 0; c < 9; c++) fft3_field(&grid[(long)c * N], n1, n2, n3, pf[0], pf[1], pf[2]);
#pragma omp parallel for schedule(static)
        for (long v = 0; v < N; v++) {
            if (v == 0) { for (int c = 0; c < 9; c++) grid[(long)c * N] = 0.0; continue; }
            cplx a[9], r[9];
            for (int c = 0; c < 9; c++) a[c] = grid[(long)c * N + v];
            const double* g = &Goper[81 * v];
            for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) {
                cplx s(0., 0.);
                for (int k = 0; k < 3; k++) for (int l = 0; l < 3; l++) s += g[((i * 3 + j) * 3 + k) * 3 + l] * a[k * 3 + l];
                r[i * 3 + j] = s;
            }
            for (int c = 0; c < 9; c++) grid[(long)c * N + v] = r[c];
        }
        for (int c = 0; c < 9; c++) fft3_field(&grid[(long)c * N], n1, n2, n3, pb[0], pb[1], pb[2]);
        for (long v = 0; v < N; v++)
            for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) vox[v].dvelgradref[i][j] = grid[(long)(i * 3 + j) * N + v].real() / (double)N;
    }

    // ------------------------------------------------------------ correction_to_current (various_functions.f90:1062-1139)
    void correction_to_current() {
        M3 fl = {};
        for (long v = 0; v < N; v++) {
            M3 t;
            matmul3(vox[v].dvelgradref, vox[v].Finv, t);
            for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) fl[i][j] = fl[i][j] + vox[v].wgtc * t[i][j];
        }
        M3 dinv, d, du;
        if (inv3(defgradinvavgc, dinv) != 0) throw SolveError("Singular matrix in lu_inverse (correction_to_current)", -3);
        for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) d[i][j] = dvelgradavg[i][j] - fl[i][j];
        matmul3(d, dinv, du);
        M3 va = {}, vg = {}, vs = {};
        for (long v = 0; v < N; v++) {
            Voxel& x = vox[v];
            M3 t, u;
            for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) t[i][j] = x.dvelgradref[i][j] + du[i][j];
            matmul3(t, x.Finv, u);
            for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) {
                x.velgrad[i][j] = x.velgrad[i][j] + u[i][j];
                va[i][j] += x.velgrad[i][j] * x.wgtc;
                if (x.gas) vg[i][j] += x.velgrad[i][j] * x.wgtc;
                else vs[i][j] += x.velgrad[i][j] * x.wgtc;
            }
        }
        if (wphcgas > 0.0) for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) vg[i][j] /= wphcgas;
        for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) vs[i][j] /= wphcsol;
        copy3(va, velgradavg); copy3(vg, velgradavggas); copy3(vs, velgradavgsol);
    }

    // ------------------------------------------------------------ plastic_strain_rate (various_functions.f90:1367-1419)
    static void plastic_strain_rate(const double sg[6], const Phase& ph, const double (*sch)[5], const double (*trialtau)[2],
                                    double* gamdot, double edotp[6], double d[6][6]) {
        for (int i = 0; i < 6; i++) { edotp[i] = 0.0; for (int j = 0; j < 6; j++) d[i][j] = 0.0; }
        for (int is = 0; is < ph.nsyst; is++) {
            double rss = sch[is][0] * sg[0] + sch[is][1] * sg[1] + sch[is][2] * sg[2] + sch[is][3] * sg[3] + sch[is][4] * sg[4];
            int isign = (rss - 0.0 < 0.0) ? 1 : 0;  // kin(is) is identically zero
            rss = (rss - 0.0) / trialtau[is][isign];
            double dum = ph.gamd0[is] * std::pow(std::fabs(rss), ph.nrs[is] - 1);
            double rss1 = ph.nrs[is] * dum / trialtau[is][isign];
            double rss2 = rss * dum;
            gamdot[is] = rss2;
            for (int jj = 0; jj < 5; jj++) {
                edotp[jj] = edotp[jj] + sch[is][jj] * rss2;
                for (int ii = 0; ii < 5; ii++) d[ii][jj] = d[ii][jj] + sch[is][ii] * sch[is][jj] * rss1;
            }
        }
    }

    // ------------------------------------------------------------ harden (various_functions.f90:1439-1491)
    void harden(const Voxel& x, double tau[NSYSMX][2], double& gamma1) const {
        harden_rates(phase[x.phase - 1], x.gamdot, x.gacumgr, x.crss, process[ipr - 1].tdot, tau, gamma1);
    }
    // the same on explicit arguments: slip rates, accumulated shear and committed resistances
    static void harden_rates(const Phase& ph, const double* gamdot, double gamma0, const double (*crss)[2], double tdot,
                             double tau[NSYSMX][2], double& gamma1) {
        double deltgam = 0.0;
        for (int is = 0; is < ph.nsyst; is++) deltgam = deltgam + std::fabs(gamdot[is]) * tdot;
        gamma1 = gamma0 + deltgam;
        int is = 0, islast = 0;
        std::memset(tau, 0, sizeof(double) * NSYSMX * 2);
        for (int mode = 0; mode < ph.nmodes; mode++) {
            islast = islast + ph.nsm[mode];
            double tau1 = ph.tau[islast - 1][2], thet0 = ph.thet[islast - 1][0], thet1 = ph.thet[islast - 1][1];
            double fact = std::fabs(thet0 / tau1);
            double exp0 = std::exp(-fact * gamma0), exp1 = std::exp(-fact * gamma1);
            double voce = deltgam * thet1 + tau1 * (exp0 - exp1) + thet1 * (gamma0 * exp0 - gamma1 * exp1);
            for (int ism = 0; ism < ph.nsm[mode]; ism++) {
                double dtau = 0.;
                for (int js = 0; js < ph.nsyst; js++) dtau = dtau + ph.hard[is][js] * std::fabs(gamdot[js]);
                tau[is][0] = crss[is][0] + dtau * voce * tdot / deltgam;
                tau[is][1] = crss[is][1] + dtau * voce * tdot / deltgam;
                is++;
            }
        }
    }

    // ------------------------------------------------------------ solve_res (various_functions.f90:1142-1364)
    void solve_res() {
        const Process& pr = P();
        const int itmaxal = 100, itmaxaltau = 10;
        std::vector<double> es(N, 0.0), ee(N, 0.0);
        bool failed = false;
#pragma omp parallel for schedule(dynamic, 64)
        for (long v = 0; v < N; v++) {
            Voxel& x = vox[v];
            double lambda[6], sg[6], sgt[6], vs[6], edotth[6] = {0, 0, 0, 0, 0, 0};
            M3 vsym;
            t2_to_b6(x.sg, lambda);
            for (int i = 0; i < 6; i++) sg[i] = lambda[i];
            t2_to_b6(x.sgt, sgt);
            sym33(x.velgrad, vsym);
            t2_to_b6(vsym, vs);
            if (!x.gas) {
                const Phase& ph = phase[x.phase - 1];
                bool thermo = (imicro == 1 && pr.ithermo == 1);
                if (thermo) t2_to_b6(x.eth, edotth);
                double sgnorm = norm2v(sg, 6);
                double taunrm = norm2v(&x.trialtau[0][0], NSYSMX * 2);
                double tolt = std::max(pr.error, pr.erroral);
                int itertau = 0;
                double errtau = 2.0 * tolt;
                double edotp[6], dedotp[6][6], edot[6], dedot[6][6], res[6], sgold[6] = {0, 0, 0, 0, 0, 0};
                double dsgnorm = 0, ddgnorm = 0;
                while (itertau < itmaxaltau && errtau > tolt) {
                    itertau++;
                    int iterNR = 0;
                    double erral = 2.0 * pr.erroral, resoldn = 1.0;
                    while (iterNR < itmaxal && erral > pr.erroral) {
                        iterNR++;
                        int icut = 0;
                        double resn = 2.0 * resoldn;
                        while (resn > resoldn && icut < 10) {
                            plastic_strain_rate(sg, ph, x.sch, x.trialtau, x.gamdot, edotp, dedotp);
                            double ds[6];
                            for (int i = 0; i < 6; i++) ds[i] = (sg[i] - sgt[i]) / pr.tdot;
                            for (int i = 0; i < 6; i++) {
                                double s = 0; for (int j = 0; j < 6; j++) s += x.sg66[i][j] * ds[j];
                                edot[i] = edotp[i] + s;
                                for (int j = 0; j < 6; j++) dedot[i][j] = dedotp[i][j] + x.sg66[i][j] / pr.tdot;
                            }
                            if (thermo) for (int i = 0; i < 6; i++) edot[i] = edot[i] + edotth[i];
                            double e2[6];
                            for (int i = 0; i < 6; i++) e2[i] = edot[i] - vs[i];
                            for (int i = 0; i < 6; i++) {
                                double s = 0; for (int j = 0; j < 6; j++) s += x.c066mod[i][j] * e2[j];
                                res[i] = sg[i] - lambda[i] + s;
                            }
                            if (modAL) {
                                double r2[6];
                                for (int i = 0; i < 6; i++) { double s = 0; for (int j = 0; j < 6; j++) s += x.cG[i][j] * (sg[j] - lambda[j]); r2[i] = s; }
                                for (int i = 0; i < 6; i++) res[i] = res[i] - r2[i];
                            }
                            resn = norm2v(res, 6);
                            if (iterNR == 1) resoldn = resn;
                            if (resn > resoldn) for (int i = 0; i < 6; i++) sg[i] = sgold[i] + (sg[i] - sgold[i]) * 0.5;
                            icut++;
                        }
                        resoldn = resn;
                        for (int i = 0; i < 6; i++) sgold[i] = sg[i];
                        double J[36];
                        for (int i = 0; i < 6; i++) for (int j = 0; j < 6; j++) {
                            double s = 0; for (int k = 0; k < 6; k++) s += x.c066mod[i][k] * dedot[k][j];
                            J[i * 6 + j] = (i == j ? 1.0 : 0.0) + s;
                            if (modAL) J[i * 6 + j] -= x.cG[i][j];
                        }
                        if (lu_eqsystem(J, res, 6) != 0) { failed = true; }
                        for (int i = 0; i < 6; i++) sg[i] = sg[i] - res[i];
                        double a = 0, b = 0, c = 0;
                        for (int i = 0; i < 6; i++) {
                            a += (sg[i] - sgold[i]) * (sg[i] - sgold[i]);
                            b += (sg[i] - lambda[i]) * (sg[i] - lambda[i]);
                            c += (edot[i] - vs[i]) * (edot[i] - vs[i]);
                        }
                        dsgnorm = b; ddgnorm = c;
                        erral = std::sqrt(a) / sgnorm;
                    }
                    if (pr.iuphard == 1) {
                        double told[NSYSMX][2], tnew[NSYSMX][2], gac;
                        std::memcpy(told, x.trialtau, sizeof(told));
                        harden(x, tnew, gac);
                        double s = 0;
                        for (int i = 0; i < NSYSMX; i++) for (int c2 = 0; c2 < 2; c2++) s += (told[i][c2] - tnew[i][c2]) * (told[i][c2] - tnew[i][c2]);
                        errtau = std::sqrt(s) / taunrm;
                        std::memcpy(x.trialtau, tnew, sizeof(tnew));
                    } else {
                        errtau = 0.;
                    }
                }
                b6_to_t2(sg, x.sg);
                b6_to_t2(edotp, x.edotp);
                es[v] = dsgnorm * x.wgtc;
                ee[v] = ddgnorm * x.wgtc;
            } else {
                double t[6], res[6];
                for (int i = 0; i < 6; i++) t[i] = vs[i] + sgt[i] / pr.tdot * complgas;
                for (int i = 0; i < 6; i++) { double s = 0; for (int j = 0; j < 6; j++) s += x.c066mod[i][j] * t[j]; res[i] = lambda[i] + s; }
                if (modAL) for (int i = 0; i < 6; i++) { double s = 0; for (int j = 0; j < 6; j++) s += x.cG[i][j] * lambda[j]; res[i] -= s; }
                for (int i = 0; i < 6; i++) { double s = 0; for (int j = 0; j < 6; j++) s += x.cgas[i][j] * res[j]; sg[i] = s; }
                b6_to_t2(sg, x.sg);
                std::memset(x.edotp, 0, sizeof(M3));
                for (int i = 0; i < NSYSMX; i++) x.gamdot[i] = 0.0;
            }
        }
        if (failed) throw SolveError("Failed system solve in lu_eqsystem (solve_res)", -3);
        erre = 0.0; errs = 0.0;
        for (long v = 0; v < N; v++) { errs += es[v]; erre += ee[v]; }
        if (erre < 0 || errs < 0) throw SolveError("ERRE/ERRS negative -> convergence failed!", -4);
        erre = std::sqrt(erre);
        errs = std::sqrt(errs);
    }

    // ------------------------------------------------------------ state_6x6_evpsc (various_functions.f90:1638-1705)
    void state_6x6(const int idsim[6], double dbar[6], const int iscau[6], double sbar[6], const M6 xm, const double devp0[6],
                   M3 scauchy, M3 dsim) {
        double profac[6], dbarv[6], sbarv[6], devp0v[6], aux6[6], aux6a[6];
        for (int i = 1; i <= 6; i++) profac[i - 1] = 1.0 + (i / 4);
        t2_to_voigt(dsim, dbarv);
        t2_to_voigt(scauchy, sbarv);
        T4 a4;
        M6 xmv;
        b66_to_t4(xm, a4);
        t4_to_v66(a4, xmv);
        M3 a33;
        b6_to_t2(devp0, a33);
        t2_to_voigt(a33, devp0v);
        for (int i = 0; i < 6; i++) aux6[i] = dbarv[i] - devp0v[i];
        double A[36];
        for (int i = 0; i < 6; i++) {
            aux6a[i] = -1.0 * idsim[i] * aux6[i];
            for (int j = 0; j < 6; j++) {
                aux6a[i] = aux6a[i] + xmv[i][j] * iscau[j] * sbarv[j] * profac[j];
                A[i * 6 + j] = iscau[j] * (i == j ? 1 : 0) - idsim[j] * xmv[i][j] * profac[j];
            }
        }
        if (lu_eqsystem(A, aux6a, 6) != 0) throw SolveError("Failed system solve in lu_eqsystem (state_6x6_evpsc)", -3);
        for (int i = 0; i < 6; i++) {
            aux6[i] = idsim[i] * aux6[i] + iscau[i] * aux6a[i];
            sbarv[i] = iscau[i] * sbarv[i] + idsim[i] * aux6a[i];
        }
        for (int i = 0; i < 6; i++) dbarv[i] = aux6[i] + devp0v[i];
        voigt_to_t2(dbarv, dsim);
        t2_to_b6(dsim, dbar);
        voigt_to_t2(sbarv, scauchy);
        t2_to_b6(scauchy, sbar);
    }

    // ------------------------------------------------------------ calc_velgradavg_corr (various_functions.f90:1526-1635)
    void calc_velgradavg_corr() {
        Process& pr = P();
        M3 ss = {}, sa = {};
        for (long v = 0; v < N; v++) {
            const Voxel& x = vox[v];
            if (x.gas) continue;
            for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) {
                ss[i][j] = ss[i][j] + x.wgtc * x.sg[i][j];
                sa[i][j] = sa[i][j] + x.wgtc * x.sg[i][j];
            }
        }
        for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) ss[i][j] /= wphcsol;
        copy3(sa, sgavg);
        copy3(ss, sgavgsol);
        svmavg = vm_stress(sgavg);
        M3 a33 = {};
        for (int i = 0; i < 6; i++) {
            int ii = IJV[i][0], jj = IJV[i][1];
            a33[ii][jj] = pr.iscau[i] * (pr.scauchy[ii][jj] - sgavg[ii][jj]);
            a33[jj][ii] = pr.iscau[i] * (pr.scauchy[jj][ii] - sgavg[jj][ii]);
        }
        errsbc = frob3(a33);
        M3 vsym, vasym;
        sym33(velgradavg, vsym);
        antisym33(velgradavg, vasym);
        double dbar[6], sbar[6], devp0[6];
        t2_to_b6(vsym, dbar);
        t2_to_b6(sgavg, sbar);
        M6 mev;
        t4_to_b66(de_ds, mev);
        for (int i = 0; i < 6; i++) { double s = 0; for (int j = 0; j < 6; j++) s += mev[i][j] * sbar[j]; devp0[i] = dbar[i] - s; }
        state_6x6(pr.idsim, dbar, pr.iscau, sbar, mev, devp0, pr.scauchy, pr.dsim);
        M3 dsym, w = {}, dasym;
        for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) dsym[i][j] = pr.dsim[i][j] - vsym[i][j];
        for (int ii = 0; ii < 3; ii++)
            for (int jj = 0; jj < 3; jj++) {
                if (ii == jj) { w[ii][jj] = 0.0; continue; }
                if (pr.iudot[ii][jj] == 1 && pr.iudot[jj][ii] == 0) {
                    w[ii][jj] = pr.udot[ii][jj] - pr.dsim[ii][jj];
                    w[jj][ii] = -w[ii][jj];
                } else if (pr.iudot[ii][jj] == 0 && pr.iudot[jj][ii] == 1) {
                    // already assigned
                } else if (pr.iudot[ii][jj] == 1 && pr.iudot[jj][ii] == 1) {
                    w[ii][jj] = 0.5 * (pr.udot[ii][jj] - pr.udot[jj][ii]);
                } else {
                    w[jj][ii] = 0.0;
                }
            }
        for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) dasym[i][j] = w[i][j] - vasym[i][j];
        for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) dvelgradavg[i][j] = dsym[i][j] + dasym[i][j];
    }

    // ------------------------------------------------------------ update_plastic_defgrad (various_functions.f90:1748-1827)
    void update_plastic_defgrad() {
        double tdot = P().tdot;
        bool failed = false;
#pragma omp parallel for schedule(static)
        for (long v = 0; v < N; v++) {
            Voxel& x = vox[v];
            if (x.gas) continue;
            const Phase& ph = phase[x.phase - 1];
            M3 Lp = {};
            for (int is = 0; is < ph.nsyst; is++) {
                double dn[3], db[3];
                for (int i = 0; i < 3; i++) {
                    dn[i] = x.ag[i][0] * ph.dnca[is][0] + x.ag[i][1] * ph.dnca[is][1] + x.ag[i][2] * ph.dnca[is][2];
                    db[i] = x.ag[i][0] * ph.dbca[is][0] + x.ag[i][1] * ph.dbca[is][1] + x.ag[i][2] * ph.dbca[is][2];
                }
                for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) Lp[i][j] = Lp[i][j] + db[i] * dn[j] * x.gamdot[is];
            }
            M3 d, e;
            for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) d[i][j] = Lp[i][j] * tdot;
            if (expm_adaptive(d, e) != 0) failed = true;
            matmul3(e, x.Fp, x.Fp);
        }
        if (failed) throw SolveError("Singular (V-U) in matrix_exp_pade", -3);
    }

    // ------------------------------------------------------------ integrate_tensor2 + cell2node + xnode (various_functions.f90:1970-2056)
    void update_grid_velgrad_node() {
        double tdot = P().tdot;
        int ideriv = P().igamma;
        std::vector<cplx> g9(9 * N), g3(3 * N);
        M3 vavg = {};
        for (long v = 0; v < N; v++) {
            M3 t;
            matmul3(vox[v].velgrad, vox[v].F, t);
            for (int l = 0; l < 3; l++) for (int m = 0; m < 3; m++) g9[(long)(l * 3 + m) * N + v] = cplx(t[l][m], 0.0);
            for (int l = 0; l < 3; l++) for (int m = 0; m < 3; m++) vavg[l][m] = vavg[l][m] + t[l][m] * wgt;
        }
        for (int c = 0; c < 9; c++) fft3_field(&g9[(long)c * N], n1, n2, n3, pf[0], pf[1], pf[2]);
        for (long v = 0; v < N; v++) {
            int i = (int)(v % n1) + 1, j = (int)((v / n1) % n2) + 1, k = (int)(v / ((long)n1 * n2)) + 1;
            double xk[3];
            spatial_freq(i, j, k, xk);
            cplx km[3];
            if (ideriv == 2) {
                cplx base = cplx(0.0, 1.0) * 0.25 * (1.0 + std::exp(cplx(0.0, xk[0]))) * (1.0 + std::exp(cplx(0.0, xk[1]))) *
                            (1.0 + std::exp(cplx(0.0, xk[2])));
                for (int l = 0; l < 3; l++) km[l] = std::tan(xk[l] / 2.0) * base;
            } else {
                for (int l = 0; l < 3; l++) km[l] = (ideriv == 0) ? cplx(0.0, xk[l]) : cplx(0.0, std::sin(xk[l]));
            }
            cplx kk = std::conj(km[0]) * km[0] + std::conj(km[1]) * km[1] + std::conj(km[2]) * km[2];
            if (kk.real() > 0.0) {
                for (int l = 0; l < 3; l++) {
                    cplx s(0.0, 0.0);
                    for (int m = 0; m < 3; m++) s = s + std::conj(km[m]) * g9[(long)(l * 3 + m) * N + v] / kk;
                    g3[(long)l * N + v] = s;
                }
            } else {
                for (int l = 0; l < 3; l++) g3[(long)l * N + v] = 0.0;
            }
            if ((n1 % 2 == 0 && i == n1 / 2 + 1) && (n2 % 2 == 0 && j == n2 / 2 + 1) && ((n3 % 2 == 0 && k == n3 / 2 + 1) && n3 > 1) && ideriv == 2)
                for (int l = 0; l < 3; l++) g3[(long)l * N + v] = 0.0;
        }
        for (int c = 0; c < 3; c++) fft3_field(&g3[(long)c * N], n1, n2, n3, pb[0], pb[1], pb[2]);
        std::vector<double> dv(3 * N);
        for (long v = 0; v < N; v++)
            for (int l = 0; l < 3; l++) dv[3 * v + l] = g3[(long)l * N + v].real() / (double)N;
        long nn1 = n1 + 1, nn2 = n2 + 1, nn3 = n3 + 1;
        std::vector<double> dn(3 * nn1 * nn2 * nn3);
        if (ideriv != 2) {
            for (int k = 1; k <= n3 + 1; k++) {
                int k1 = k - 1, k2 = k; if (k1 == 0) k1 = n3; if (k2 == n3 + 1) k2 = 1;
                for (int j = 1; j <= n2 + 1; j++) {
                    int j1 = j - 1, j2 = j; if (j1 == 0) j1 = n2; if (j2 == n2 + 1) j2 = 1;
                    for (int i = 1; i <= n1 + 1; i++) {
                        int i1 = i - 1, i2 = i; if (i1 == 0) i1 = n1; if (i2 == n1 + 1) i2 = 1;
                        auto c = [&](int a, int b, int cc, int l) { return dv[3 * vidx(a - 1, b - 1, cc - 1) + l]; };
                        for (int l = 0; l < 3; l++)
                            dn[3 * ((i - 1) + nn1 * ((j - 1) + nn2 * (k - 1))) + l] =
                                (c(i2, j2, k2, l) + c(i1, j2, k2, l) + c(i2, j1, k2, l) + c(i2, j2, k1, l) + c(i1, j1, k2, l) +
                                 c(i1, j2, k1, l) + c(i2, j1, k1, l) + c(i1, j1, k1, l)) * 0.125;
                    }
                }
            }
        } else {
            for (int k = 0; k < nn3; k++) for (int j = 0; j < nn2; j++) for (int i = 0; i < nn1; i++)
                for (int l = 0; l < 3; l++)
                    dn[3 * (i + nn1 * (j + nn2 * k)) + l] = dv[3 * vidx(i % n1, j % n2, k % n3) + l];
        }
        for (int k = 0; k < n3node; k++)
            for (int j = 0; j < n2 + 1; j++)
                for (int i = 0; i < n1 + 1; i++) {
                    double xx[3] = {(double)(i + 1) - 0.5, (double)(j + 1) - 0.5, (n3node == 1) ? 0.0 : (double)(k + 1) - 0.5};
                    long p = 3L * (i + (long)(n1 + 1) * (j + (long)(n2 + 1) * k));
                    long q = 3L * (i + nn1 * (j + nn2 * k));
                    for (int l = 0; l < 3; l++) {
                        double s = vavg[l][0] * xx[0] + vavg[l][1] * xx[1] + vavg[l][2] * xx[2];
                        xnode[p + l] = xnode[p + l] + (s + dn[q + l]) * tdot;
                    }
                }
    }

    // ------------------------------------------------------------ update_defgrad (various_functions.f90:2152-2282)
    void update_defgrad() {
        double tdot = P().tdot;
        bool failed = false;
#pragma omp parallel for schedule(static)
        for (long v = 0; v < N; v++) {
            Voxel& x = vox[v];
            M3 d, e, Fo;
            copy3(x.F, Fo);
            for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) d[i][j] = x.velgrad[i][j] * tdot;
            if (expm_adaptive(d, e) != 0) failed = true;
            matmul3(e, Fo, x.F);
            x.detF = det33(x.F);
            if (x.detF < 0.0 && verbose) std::printf(" -> WARNING: detF=%13.6E in voxel (%ld)\n", x.detF, v);
            if (inv3(x.F, x.Finv) != 0) failed = true;
            copy3(e, x.Finc);
            x.wgtc = wgt * x.detF;
        }
        if (failed) throw SolveError("Singular matrix in lu_inverse (update_defgrad)", -3);
        M3 fa = {}, fc = {}, fcs = {}, fcg = {};
        double ws = 0, wg = 0, dav = 0;
        for (long v = 0; v < N; v++) {
            const Voxel& x = vox[v];
            for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) {
                fa[i][j] = fa[i][j] + x.F[i][j] * wgt;
                fc[i][j] = fc[i][j] + x.Finv[i][j] * wgt * x.detF;
                if (x.gas) fcg[i][j] = fcg[i][j] + x.Finv[i][j] * wgt * x.detF;
                else fcs[i][j] = fcs[i][j] + x.Finv[i][j] * wgt * x.detF;
            }
            if (x.gas) wg = wg + wgt * x.detF;
            else ws = ws + wgt * x.detF;
            dav = dav + x.detF * wgt;
        }
        copy3(fa, defgradavg);
        for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) fc[i][j] /= dav;
        copy3(fc, defgradinvavgc);
        wphcsol = ws / dav;
        wphcgas = wg / dav;
        for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) defgradinvavgcs[i][j] = fcs[i][j] / dav / wphcsol;
        if (wphcgas > 0.0) { for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) defgradinvavgcg[i][j] = fcg[i][j] / dav / wphcgas; }
        else eye3(defgradinvavgcg);
        for (long v = 0; v < N; v++) vox[v].wgtc = vox[v].wgtc / dav;
    }

    // ------------------------------------------------------------ update_elstic_defgrad (various_functions.f90:2285-2324)
    void update_elastic_defgrad() {
        bool failed = false;
#pragma omp parallel for schedule(static)
        for (long v = 0; v < N; v++) {
            Voxel& x = vox[v];
            if (x.gas) continue;
            M3 feinv, fpf, fpfinv;
            if (inv3(x.Fe, feinv) != 0) failed = true;
            matmul3(x.Fp, x.Fini, fpf);
            if (inv3(fpf, fpfinv) != 0) failed = true;
            matmul3(x.F, fpfinv, x.Fe);
            matmul3(x.Fe, feinv, x.Feinc);
        }
        if (failed) throw SolveError("Singular matrix in lu_inverse (update_elstic_defgrad)", -3);
    }

    // ------------------------------------------------------------ update_el_stiff (various_functions.f90:2327-2402)
    void update_el_stiff() {
        bool failed = false;
#pragma omp parallel for schedule(static)
        for (long v = 0; v < N; v++) {
            Voxel& x = vox[v];
            if (x.gas) continue;
            M3 aa;
            matmul3(x.Fe, x.ag, aa);
            double detFe = det33(x.Fe);
            T4 c;
            rotate4(aa, phase[x.phase - 1].C, c);
            for (int i = 0; i < 81; i++) (&c[0][0][0][0])[i] /= detFe;
            t4_to_b66(c, x.cg66);
            if (inv6(x.cg66, x.sg66) != 0) failed = true;
        }
        if (failed) throw SolveError("Singular matrix in lu_inverse (update_el_stiff)", -3);
    }

    // ------------------------------------------------------------ update_tensor_config (various_functions.f90:2405-2492)
    void update_tensor_config() {
        bool failed = false;
#pragma omp parallel for schedule(static)
        for (long v = 0; v < N; v++) {
            Voxel& x = vox[v];
            double detei = det33(x.Feinc);
            M3 finv;
            if (inv3(x.Finc, finv) != 0) failed = true;
            if (!x.gas) {
                M3 R, U, Rt, t;
                polar(x.Finc, R, U);
                transpose3(R, Rt);
                matmul3(R, x.disgradsym, t); matmul3(t, Rt, x.disgradsym);
                matmul3(R, x.ept, t); matmul3(t, Rt, x.ept);
                M3 Ft;
                transpose3(x.Feinc, Ft);
                matmul3(x.Feinc, x.sgt, t); matmul3(t, Ft, x.sgt);
                for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) x.sgt[i][j] /= detei;
            }
            matmul3(x.velgrad, finv, x.velgrad);
        }
        if (failed) throw SolveError("Singular matrix in lu_inverse (update_tensor_config)", -3);
        M3 va = {};
        for (long v = 0; v < N; v++)
            for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) va[i][j] = va[i][j] + vox[v].velgrad[i][j] * vox[v].wgtc;
        M3 dinv, d, du;
        if (inv3(defgradinvavgc, dinv) != 0) throw SolveError("Singular matrix in lu_inverse (update_tensor_config)", -3);
        for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) d[i][j] = velgradavg[i][j] - va[i][j];
        matmul3(d, dinv, du);
#pragma omp parallel for schedule(static)
        for (long v = 0; v < N; v++) {
            M3 t;
            matmul3(du, vox[v].Finv, t);
            for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) vox[v].velgrad[i][j] = vox[v].velgrad[i][j] + t[i][j];
        }
    }

    // ------------------------------------------------------------ update_hardening (various_functions.f90:1493-1523)
    void update_hardening() {
#pragma omp parallel for schedule(static)
        for (long v = 0; v < N; v++) {
            Voxel& x = vox[v];
            if (x.gas) continue;
            double t[NSYSMX][2], g;
            harden(x, t, g);
            std::memcpy(x.crss, t, sizeof(t));
            std::memcpy(x.trialtau, t, sizeof(t));
            x.gacumgr = g;
        }
    }

    // ------------------------------------------------------------ calc_c0 (various_functions.f90:2537-2649)
    void calc_c0() {
        const Process& pr = P();
        M6 dP = {};
        T4 dsde = {};
        bool failed = false;
        std::vector<double> part(N * (81 + 36));
#pragma omp parallel for schedule(static)
        for (long v = 0; v < N; v++) {
            const Voxel& x = vox[v];
            if (x.gas) continue;
            const Phase& ph = phase[x.phase - 1];
            double sg6[6], sgt6[6], edotp6[6], dp[6][6], gd[NSYSMX];
            t2_to_b6(x.sg, sg6);
            t2_to_b6(x.sgt, sgt6);
            plastic_strain_rate(sg6, ph, x.sch, x.trialtau, gd, edotp6, dp);
            M6 tr, tri;
            for (int i = 0; i < 6; i++) for (int j = 0; j < 6; j++) tr[i][j] = x.sg66[i][j] / pr.tdot * pr.tdot / pr.tdotref + dp[i][j];
            if (inv6(tr, tri) != 0) failed = true;
            T4 dsg, dPg;
            b66_to_t4(tri, dsg);
            for (int l = 0; l < 3; l++) for (int k = 0; k < 3; k++) for (int j = 0; j < 3; j++) for (int i = 0; i < 3; i++) {
                double s = 0.0;
                for (int m = 0; m < 3; m++) for (int n = 0; n < 3; n++) s = s + dsg[i][m][k][n] * x.Finv[j][m] * x.Finv[l][n] * x.detF;
                dPg[i][j][k][l] = s;
            }
            M6 dP6;
            t4_to_b66(dPg, dP6);
            double* pp = &part[v * 117];
            for (int c = 0; c < 81; c++) pp[c] = (&dsg[0][0][0][0])[c] * x.wgtc;
            for (int c = 0; c < 36; c++) pp[81 + c] = (&dP6[0][0])[c] * wgt;
        }
        if (failed) throw SolveError("Singular matrix in lu_inverse (calc_c0)", -3);
        for (long v = 0; v < N; v++) {
            if (vox[v].gas) continue;
            const double* pp = &part[v * 117];
            for (int c = 0; c < 81; c++) (&dsde[0][0][0][0])[c] += pp[c];
            for (int c = 0; c < 36; c++) (&dP[0][0])[c] += pp[81 + c];
        }
        for (int c = 0; c < 81; c++) (&dsde[0][0][0][0])[c] /= wphcsol;
        for (int c = 0; c < 36; c++) (&dP[0][0])[c] /= wphsol;
        M6 a, ai;
        t4_to_b66(dsde, a);
        if (inv6(a, ai) != 0) throw SolveError("Singular matrix in lu_inverse (calc_c0)", -3);
        b66_to_t4(ai, de_ds);
        for (int i = 0; i < 6; i++) for (int j = 0; j < 6; j++) { c066[i][j] = dP[i][j] * pr.xc0; a[i][j] = dP[i][j] * pr.xc0; }
        if (inv6(a, ai) != 0) throw SolveError("Singular matrix in lu_inverse (calc_c0)", -3);
        b66_to_t4(c066, c0);
        b66_to_t4(ai, s0);
    }

    // ------------------------------------------------------------ kinematic_increments (various_functions.f90:2766-2837)
    void stretch_rot(const M3 Finc, double& volinc, double& rotang, double& stretchinc, bool cof_det, double* Jinc_out) const {
        double Jinc = cof_det ? det33_cof(Finc) : det33(Finc);
        if (Jinc_out) *Jinc_out = Jinc;
        volinc = std::fabs(std::log(std::max(Jinc, TINY)));
        M3 R, U;
        polar(Finc, R, U);
        double arg = 0.5 * ((R[0][0] + R[1][1] + R[2][2]) - 1.0);
        arg = std::max(-1.0, std::min(1.0, arg));
        rotang = std::acos(arg) * 180 / PI;
        double w[3];
        M3 Q, t, lu;
        sym_eig3(U, w, Q);
        for (int ii = 0; ii < 3; ii++) { double lw = std::log(std::max(w[ii], TINY)); for (int r = 0; r < 3; r++) t[r][ii] = Q[r][ii] * lw; }
        M3 Qt;
        transpose3(Q, Qt);
        matmul3(t, Qt, lu);
        stretchinc = frob3(lu);
    }
    int kinematic_substep(double tdot_step, double& mv, double& mr, double& ms, double& mdet) {
        mv = 0; mr = 0; ms = 0; mdet = HUGE_;
        std::vector<double> a(4 * N);
        bool failed = false;
#pragma omp parallel for schedule(static)
        for (long v = 0; v < N; v++) {
            M3 L, Fi;
            for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) L[i][j] = vox[v].velgrad[i][j] * tdot_step;
            if (expm_adaptive(L, Fi) != 0) failed = true;
            double vi, ro, st, Ji;
            stretch_rot(Fi, vi, ro, st, false, &Ji);
            a[4 * v] = vi; a[4 * v + 1] = ro; a[4 * v + 2] = st; a[4 * v + 3] = vox[v].detF * Ji;
        }
        if (failed) throw SolveError("Singular (V-U) in matrix_exp_pade", -3);
        for (long v = 0; v < N; v++) {
            mv = std::max(mv, a[4 * v]); mr = std::max(mr, a[4 * v + 1]); ms = std::max(ms, a[4 * v + 2]); mdet = std::min(mdet, a[4 * v + 3]);
        }
        double worst = std::max(std::max(1.0, mv / 5.0e-2), std::max(mr / 2.0, ms / 5.0e-2));
        return std::max(1, (int)std::ceil(worst));
    }

    // ------------------------------------------------------------ take_snapshot / rollback (various_functions.f90:2839-2895)
    void take_snapshot() {
        copy3(P().dsim, P().dsim_snapshot);
        copy3(P().scauchy, P().scauchy_snapshot);
        for (long v = 0; v < N; v++) {
            Voxel& x = vox[v];
            copy3(x.velgrad, x.s_velgrad); copy3(x.velgradold, x.s_velgradold); copy3(x.sg, x.s_sg); copy3(x.edotp, x.s_edotp);
            std::memcpy(x.s_gamdot, x.gamdot, sizeof(x.gamdot));
            std::memcpy(x.s_trialtau, x.trialtau, sizeof(x.trialtau));
        }
    }
    void rollback() {
        copy3(P().dsim_snapshot, P().dsim);
        copy3(P().scauchy_snapshot, P().scauchy);
        for (long v = 0; v < N; v++) {
            Voxel& x = vox[v];
            copy3(x.s_velgrad, x.velgrad); copy3(x.s_velgradold, x.velgradold); copy3(x.s_sg, x.sg); copy3(x.s_edotp, x.edotp);
            std::memcpy(x.gamdot, x.s_gamdot, sizeof(x.gamdot));
            std::memcpy(x.trialtau, x.s_trialtau, sizeof(x.trialtau));
        }
    }

    // ------------------------------------------------------------ update_diagnostics (types.f90:345-758)
    void update_diagnostics() {
        std::vector<double> a(9 * N);
        bool scan_cond = true;
#pragma omp parallel for schedule(static)
        for (long v = 0; v < N; v++) {
            const Voxel& x = vox[v];
            double* r = &a[9 * v];
            double vi, ro, st;
            stretch_rot(x.Finc, vi, ro, st, true, nullptr);
            r[0] = vi; r[1] = ro; r[2] = st;
            M3 dl;
            for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) dl[i][j] = x.velgrad[i][j] - x.s_velgrad[i][j];
            r[3] = frob3(dl);
            r[4] = frob3(x.s_velgrad);
            r[5] = scan_cond ? cond1_est_6x6(x.c066mod) : 0.0;
            r[6] = (scan_cond && x.gas) ? cond1_est_6x6(x.cgas) : 0.0;
        }
        double Lref = std::max(lvmavg, TINY);
        double Lfloor = std::max(1.0e-12 * Lref, TINY);
        double dmin = HUGE_, dmin_s = HUGE_, dmin_g = HUGE_;
        int imin_s[3] = {0, 0, 0}, imin_g[3] = {0, 0, 0};
        double s2s = 0, sws = 0, mxs = 0, s2g = 0, swg = 0, mxg = 0, s2a = 0, swa = 0, mxa = 0;
        double vms = 0, vmg = 0, sms = 0, smg = 0, rms = 0, rmg = 0, ccs = 0, ccg = 0, cgg = 0;
        for (long v = 0; v < N; v++) {
            const Voxel& x = vox[v];
            const double* r = &a[9 * v];
            double denom = std::max(r[4], Lfloor);
            double rel = r[3] / denom;
            double w = x.wgtc;
            int i = (int)(v % n1) + 1, j = (int)((v / n1) % n2) + 1, k = (int)(v / ((long)n1 * n2)) + 1;
            s2a += (rel * rel) * w; swa += w; mxa = std::max(mxa, rel);
            dmin = std::min(dmin, x.detF);
            if (x.gas) {
                if (x.detF <= dmin_g) { dmin_g = x.detF; imin_g[0] = i; imin_g[1] = j; imin_g[2] = k; }
                s2g += (rel * rel) * w; swg += w; mxg = std::max(mxg, rel);
                vmg = std::max(vmg, r[0]); rmg = std::max(rmg, r[1]); smg = std::max(smg, r[2]);
                ccg = std::max(ccg, r[5]); cgg = std::max(cgg, r[6]);
            } else {
                if (x.detF <= dmin_s) { dmin_s = x.detF; imin_s[0] = i; imin_s[1] = j; imin_s[2] = k; }
                s2s += (rel * rel) * w; sws += w; mxs = std::max(mxs, rel);
                vms = std::max(vms, r[0]); rms = std::max(rms, r[1]); sms = std::max(sms, r[2]);
                ccs = std::max(ccs, r[5]);
            }
        }
        Diag& d = diag;
        d.detF_min = dmin; d.detF_min_sol = dmin_s; d.detF_min_gas = dmin_g;
        d.volinc_max_sol = vms; d.volinc_max_gas = vmg; d.stretchinc_max_sol = sms; d.stretchinc_max_gas = smg;
        d.rotang_max_sol = rms; d.rotang_max_gas = rmg;
        for (int q = 0; q < 3; q++) { d.imin_sol[q] = imin_s[q]; d.imin_gas[q] = imin_g[q]; }
        d.cond_c066mod_max_sol = ccs; d.cond_c066mod_max_gas = ccg; d.cond_cgas_max = cgg;
        if (d.detF_min >= HUGE_ * 0.5) d.detF_min = 0.0;
        if (d.detF_min_sol >= HUGE_ * 0.5) d.detF_min_sol = 0.0;
        if (d.detF_min_gas >= HUGE_ * 0.5) d.detF_min_gas = 0.0;
        d.dL_step_rms = swa > 0 ? std::sqrt(s2a / swa) : 0.0; d.dL_step_max = mxa;
        d.dL_step_rms_sol = sws > 0 ? std::sqrt(s2s / sws) : 0.0; d.dL_step_max_sol = mxs;
        d.dL_step_rms_gas = swg > 0 ? std::sqrt(s2g / swg) : 0.0; d.dL_step_max_gas = mxg;
        d.dvelgradavg_mag = frob3(dvelgradavg);
        d.detF_min_ratio = safe_ratio(d.detF_min, d.detF_min_prev);
        d.detF_min_relstep = safe_rel_change(d.detF_min, d.detF_min_prev);
        d.detF_min_prev = d.detF_min;
        d.detF_min_sol_ratio = safe_ratio(d.detF_min_sol, d.detF_min_sol_prev);
        d.detF_min_sol_relstep = safe_rel_change(d.detF_min_sol, d.detF_min_sol_prev);
        d.detF_min_sol_prev = d.detF_min_sol;
        d.detF_min_gas_ratio = safe_ratio(d.detF_min_gas, d.detF_min_gas_prev);
        d.detF_min_gas_relstep = safe_rel_change(d.detF_min_gas, d.detF_min_gas_prev);
        d.detF_min_gas_prev = d.detF_min_gas;
        d.volinc_max_sol_relstep = safe_rel_change(d.volinc_max_sol, d.volinc_max_sol_prev); d.volinc_max_sol_prev = d.volinc_max_sol;
        d.volinc_max_gas_relstep = safe_rel_change(d.volinc_max_gas, d.volinc_max_gas_prev); d.volinc_max_gas_prev = d.volinc_max_gas;
        d.stretchinc_max_sol_relstep = safe_rel_change(d.stretchinc_max_sol, d.stretchinc_max_sol_prev); d.stretchinc_max_sol_prev = d.stretchinc_max_sol;
        d.stretchinc_max_gas_relstep = safe_rel_change(d.stretchinc_max_gas, d.stretchinc_max_gas_prev); d.stretchinc_max_gas_prev = d.stretchinc_max_gas;
        d.rotang_max_sol_prev = d.rotang_max_sol;
        d.rotang_max_gas_prev = d.rotang_max_gas;
    }

    // ------------------------------------------------------------ outputs
    std::string csv(const char* name) const {
        if (!outdir.empty() && outdir.back() == '/') return outdir + name;
        return outdir + "/" + name;
    }
    void write_headers() {
        if (!write_files) return;
        FILE* f = std::fopen(csv("diagnostics.csv").c_str(), "w");
        if (!f) throw SolveError("write_diagnostics: failed to open diagnostics.csv for writing", -5);
        std::fprintf(f, "iter,macrostep,ipr,sim_time,wall_time,tdot,vm_max_inc,tdotref,erre,errs,errsbc,s33_target,s33,s33_sol,"
                        "detF_min_sol,detF_min_gas,detF_min_sol_rel,detF_min_gas_rel,volinc_max_sol,volinc_max_gas,volinc_max_sol_rel,"
                        "volinc_max_gas_rel,stretchinc_max_sol,stretchinc_max_gas,stretchinc_max_sol_rel,stretchinc_max_gas_rel,"
                        "rotang_max_sol,rotang_max_gas,dL_step_rms_sol,dL_step_rms_gas,dL_step_rms,dL_step_max_sol,dL_step_max_gas,"
                        "dL_step_max,dvelgradavg_mag,cond_c066mod_max_sol,cond_c066mod_max_gas,cond_cgas_max,imin_sol_i,imin_sol_j,"
                        "imin_sol_k,imin_gas_i,imin_gas_j,imin_gas_k\n");
        std::fclose(f);
        f = std::fopen(csv("results.csv").c_str(), "w");
        if (!f) throw SolveError("results: failed to open results.csv for writing", -5);
        std::fprintf(f, "iter,macrostep,ipr,sim_time,wall_time,tdot,tdot_ref,eav11,eav22,eav33,eav23,eav13,eav12,sav11,sav22,sav33,"
                        "sav23,sav13,sav12,epav11,epav22,epav33,epav23,epav13,epav12,eelav11,eelav22,eelav33,eelav23,eelav13,"
                        "eelav12,vgrad11,vgrad22,vgrad33,vgrad23,vgrad13,vgrad12,edotp11,edotp22,edotp33,edotp23,edotp13,edotp12,"
                        "evm,evmp,dvm,dvmp,svm,gamma,g,geff\n");
        std::fclose(f);
    }
    void write_rows(int iter_l, int imacro, int ipr_l, double stime, double wtime, double tdot, double tdotref, double gamma, double g,
                    double geff) {
        double* R = last_results;
        int c = 0;
        R[c++] = iter_l; R[c++] = imacro; R[c++] = ipr_l; R[c++] = stime; R[c++] = wtime; R[c++] = tdot; R[c++] = tdotref;
        auto put6 = [&](const M3 m) { R[c++] = m[0][0]; R[c++] = m[1][1]; R[c++] = m[2][2]; R[c++] = m[1][2]; R[c++] = m[0][2]; R[c++] = m[0][1]; };
        put6(eavg); put6(sgsolavg); put6(epavg); put6(eelavg); put6(velgradavg); put6(edotpavg);
        R[c++] = evmavg; R[c++] = evmpavg; R[c++] = dvmavg; R[c++] = dvmpavg; R[c++] = svmavg; R[c++] = gamma; R[c++] = g; R[c++] = geff;
        const Diag& d = diag;
        double* D = last_diag;
        double dv[44] = {(double)iter_l, (double)imacro, (double)ipr_l, stime, wtime, tdot, d.devm_inc_max, d.tdotref, d.erre, d.errs,
                         d.errsbc, d.s33_target, d.s33, d.s33_sol, d.detF_min_sol, d.detF_min_gas, d.detF_min_sol_relstep,
                         d.detF_min_gas_relstep, d.volinc_max_sol, d.volinc_max_gas, d.volinc_max_sol_relstep, d.volinc_max_gas_relstep,
                         d.stretchinc_max_sol, d.stretchinc_max_gas, d.stretchinc_max_sol_relstep, d.stretchinc_max_gas_relstep,
                         d.rotang_max_sol, d.rotang_max_gas, d.dL_step_rms_sol, d.dL_step_rms_gas, d.dL_step_rms, d.dL_step_max_sol,
                         d.dL_step_max_gas, d.dL_step_max, d.dvelgradavg_mag, d.cond_c066mod_max_sol, d.cond_c066mod_max_gas,
                         d.cond_cgas_max, (double)d.imin_sol[0], (double)d.imin_sol[1], (double)d.imin_sol[2], (double)d.imin_gas[0],
                         (double)d.imin_gas[1], (double)d.imin_gas[2]};
        std::memcpy(D, dv, sizeof(dv));
        if (!write_files) return;
        FILE* f = std::fopen(csv("diagnostics.csv").c_str(), "a");
        if (!f) throw SolveError("write_diagnostics: failed to open diagnostics.csv for append", -5);
        for (int q = 0; q < 44; q++) {
            bool isint = (q < 3) || q >= 38;
            if (isint) std::fprintf(f, "%d", (int)D[q]);
            else std::fprintf(f, "%s", fmt_g0(D[q]).c_str());
            std::fputc(q == 43 ? '\n' : ',', f);
        }
        std::fclose(f);
        f = std::fopen(csv("results.csv").c_str(), "a");
        if (!f) throw SolveError("write_results: failed to open results.csv for append", -5);
        for (int q = 0; q < 51; q++) {
            if (q < 3) std::fprintf(f, "%d", (int)R[q]);
            else std::fprintf(f, "%s", fmt_g0(R[q]).c_str());
            std::fputc(q == 50 ? '\n' : ',', f);
        }
        std::fclose(f);
    }
    // write_vtk_cell (IO_functions.f90:945-1235)
    void write_vtk(int istp) {
        if (!write_files) return;
        char name[64];
        std::snprintf(name, sizeof(name), "microstr_cell_fields_stp_%05d.vtk", istp);
        std::string path = outdir + "/" + name;
        FILE* f = std::fopen(path.c_str(), "w");
        if (!f) throw SolveError("ioerr in writevtk", -5);
        std::fprintf(f, "# vtk DataFile Version 3.0\nmicrostructure data\nASCII\nDATASET UNSTRUCTURED_GRID\n");
        long ncell;
        long nn1 = n1 + 1, nn2 = n2 + 1;
        auto nid = [&](int i, int j, int k) { return (long)i + nn1 * ((long)j + nn2 * (long)k); };
        if (n3 == 1) {
            long np = nn1 * nn2;
            std::fprintf(f, "POINTS%10ld double\n", np);
            for (int j = 0; j < n2 + 1; j++) for (int i = 0; i < n1 + 1; i++) {
                long p = 3 * nid(i, j, 0);
                std::fprintf(f, "%s%s%s\n", fmt_e18_8e3(xnode[p]).c_str(), fmt_e18_8e3(xnode[p + 1]).c_str(), fmt_e18_8e3(xnode[p + 2]).c_str());
            }
            ncell = (long)n1 * n2;
            std::fprintf(f, "CELLS%10ld%10ld\n", ncell, ncell * 5);
            for (int j = 0; j < n2; j++) for (int i = 0; i < n1; i++)
                std::fprintf(f, "%10d%10ld%10ld%10ld%10ld\n", 4, nid(i, j, 0), nid(i + 1, j, 0), nid(i, j + 1, 0), nid(i + 1, j + 1, 0));
            std::fprintf(f, "CELL_TYPES%10ld\n", ncell);
            for (long c = 0; c < ncell; c++) std::fprintf(f, "%5d\n", 8);
        } else {
            long np = nn1 * nn2 * (n3 + 1);
            std::fprintf(f, "POINTS%10ld double\n", np);
            for (int k = 0; k < n3 + 1; k++) for (int j = 0; j < n2 + 1; j++) for (int i = 0; i < n1 + 1; i++) {
                long p = 3 * nid(i, j, k);
                std::fprintf(f, "%s%s%s\n", fmt_e18_8e3(xnode[p]).c_str(), fmt_e18_8e3(xnode[p + 1]).c_str(), fmt_e18_8e3(xnode[p + 2]).c_str());
            }
            ncell = N;
            std::fprintf(f, "CELLS%10ld%10ld\n", ncell, ncell * 9);
            for (int k = 0; k < n3; k++) for (int j = 0; j < n2; j++) for (int i = 0; i < n1; i++)
                std::fprintf(f, "%10d%10ld%10ld%10ld%10ld%10ld%10ld%10ld%10ld\n", 8, nid(i, j, k), nid(i + 1, j, k), nid(i + 1, j + 1, k),
                             nid(i, j + 1, k), nid(i, j, k + 1), nid(i + 1, j, k + 1), nid(i + 1, j + 1, k + 1), nid(i, j + 1, k + 1));
            std::fprintf(f, "CELL_TYPES%10ld\n", ncell);
            for (long c = 0; c < ncell; c++) std::fprintf(f, "%5d\n", 12);
        }
        std::fprintf(f, "CELL_DATA%10ld\n", ncell);
        std::fprintf(f, "FIELD FieldData%10d\n", 11);
        int nsystmx = 0;
        for (auto& ph : phase) nsystmx = std::max(nsystmx, ph.nsyst);
        auto E = [&](double x) { return fmt_e18_8e3(clamp_subnormal(x)); };
        std::fprintf(f, "gamdot%3d%10ld double\n", nsystmx, ncell);
        for (long v = 0; v < N; v++) { for (int i = 0; i < nsystmx; i++) std::fputs(E(vox[v].gamdot[i]).c_str(), f); std::fputc('\n', f); }
        std::fprintf(f, "gamdot_acum%3d%10ld double\n", 1, ncell);
        for (long v = 0; v < N; v++) std::fprintf(f, "%s\n", E(vox[v].gacumgr).c_str());
        auto put9 = [&](const M3 m) { for (int c = 0; c < 3; c++) for (int r = 0; r < 3; r++) std::fputs(E(m[r][c]).c_str(), f); std::fputc('\n', f); };
        std::fprintf(f, "def_grad_p%3d%10ld double\n", 9, ncell);
        for (long v = 0; v < N; v++) put9(vox[v].Fp);
        std::fprintf(f, "stress%3d%10ld double\n", 6, ncell);
        for (long v = 0; v < N; v++) {
            const M3& s = vox[v].sg;
            std::fprintf(f, "%s%s%s%s%s%s\n", E(s[0][0]).c_str(), E(s[1][1]).c_str(), E(s[2][2]).c_str(), E(s[0][1]).c_str(), E(s[1][2]).c_str(), E(s[0][2]).c_str());
        }
        std::fprintf(f, "svm%3d%10ld double\n", 1, ncell);
        for (long v = 0; v < N; v++) std::fprintf(f, "%s\n", E(vm_stress(vox[v].sg)).c_str());
        std::fprintf(f, "def_grad%3d%10ld double\n", 9, ncell);
        for (long v = 0; v < N; v++) put9(vox[v].F);
        std::fprintf(f, "det_def_grad%3d%10ld double\n", 1, ncell);
        for (long v = 0; v < N; v++) std::fprintf(f, "%s\n", E(vox[v].detF).c_str());
        std::fprintf(f, "gr_id%3d%10ld int\n", 1, ncell);
        for (long v = 0; v < N; v++) std::fprintf(f, "%10d\n", vox[v].grain);
        std::fprintf(f, "ph_id%3d%10ld int\n", 1, ncell);
        for (long v = 0; v < N; v++) std::fprintf(f, "%10d\n", vox[v].phase);
        std::fprintf(f, "epvm%3d%10ld double\n", 1, ncell);
        for (long v = 0; v < N; v++) std::fprintf(f, "%s\n", E(vox[v].epvm).c_str());
        std::fprintf(f, "velgrad%3d%10ld double\n", 9, ncell);
        for (long v = 0; v < N; v++) put9(vox[v].velgrad);
        std::fclose(f);
    }

    // ------------------------------------------------------------ LS-EVPFFT.f90:144-182
    void open(const std::string& fft_in, const std::string& out, int mix_flag, int modal_flag) {
        outdir = out;
        if (write_files) {
            mkdir_p(outdir);
        }
        load_input(fft_in);
        initial_guess();
        write_vtk(0);
        start = std::time(nullptr);
        modAL = (modal_flag != 0);
        do_mix = (mix_flag != 0);
        std::memset(c066, 0, sizeof(M6));
        for (long v = 0; v < N; v++)
            if (!vox[v].gas)
                for (int i = 0; i < 6; i++) for (int j = 0; j < 6; j++) c066[i][j] = c066[i][j] + vox[v].cg66[i][j] * vox[v].wgtc;
        for (int i = 0; i < 6; i++) for (int j = 0; j < 6; j++) { c066[i][j] = c066[i][j] / wphcsol; c066[i][j] = c066[i][j] * process[0].tdot; }
        if (inv6(c066, s066) != 0) throw SolveError("Singular matrix in lu_inverse (initial c066)", -3);
        b66_to_t4(c066, c0);
        b66_to_t4(s066, s0);
        std::memcpy(de_ds, s0, sizeof(T4));
        write_headers();
        for (int p = 0; p < nproc; p++) total_macrosteps += process[p].nsteps;
        imacroloop = 1;
        ipr = 0;
        imicro = 0;
    }

    // One macrostep (LS-EVPFFT.f90:199-588).  Returns false once the deck is finished.
    bool macrostep() {
        while (ipr == 0 || imicro >= P().nsteps) {
            if (ipr >= nproc) { finished = true; return false; }
            ipr++;
            nconverged = 0;
            kinematic_controlled = (P().iscau[2] == 0);
            tdot_plan = P().tdot;
            proc_time_target = (double)P().nsteps * tdot_plan;
            proc_time_done = 0.0;
            imicro = 0;
        }
        Process& pr = P();
        imicro++;
        if (pr.ictrl == -1) {
            double remaining = std::max(0.0, proc_time_target - proc_time_done);
            pr.tdot = (remaining > 0.0) ? std::min(tdot_plan, remaining) : tdot_plan;
        }
        take_snapshot();
        bool did_converge = false, accept_step = false;
        if ((imicro == 1 && ipr == 1) || pr.iupdate == 1) update_schmid();
        form_G();
        calc_c066mod();
        iter = 0;
        while (!(did_converge || accept_step)) {
            if (iter == 0) {
                calc_gas_compl();
                std::memset(dvelgradavg, 0, sizeof(M3));
                edotvmmx = 0;
                mix = 1.0;
                erre = 2.0 * pr.error; errs = 2.0 * pr.error; errsbc = 2.0 * pr.error;
            }
            iter++;
            total_iters++;
            if (verbose) {
                std::printf("\rMACROSTEP=%d SimTime=%.0fs PROC=%d STEP=%d TDOT=%.0fs ITER=%d", imacroloop, sim_time, ipr, imicro, pr.tdot, iter);
                std::fflush(stdout);
            }
            // PK1 (LS-EVPFFT.f90:238-269)
            M3 sa = {};
            for (long v = 0; v < N; v++) for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) sa[i][j] = sa[i][j] + vox[v].sg[i][j] * vox[v].wgtc;
            copy3(sa, sgavg);
#pragma omp parallel for schedule(static)
            for (long v = 0; v < N; v++) {
                Voxel& x = vox[v];
                M3 d, t;
                for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) d[i][j] = x.sg[i][j] - sgavg[i][j];
                M3 fit;
                transpose3(x.Finv, fit);
                matmul3(d, fit, t);
                for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) x.sgPK1[i][j] = t[i][j] * x.detF;
            }
            convolution();
            correction_to_current();
            // mixing (LS-EVPFFT.f90:277-327)
            double s2s = 0, sws = 0, s2g = 0, swg = 0;
            double Lscale = std::max(lvmavg, TINY);
            for (long v = 0; v < N; v++) {
                Voxel& x = vox[v];
                if (!kinematic_controlled) {
                    double dl = 0;
                    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) dl += (x.velgrad[i][j] - x.velgradold[i][j]) * (x.velgrad[i][j] - x.velgradold[i][j]);
                    dl = std::sqrt(dl);
                    double rel = dl / Lscale;
                    if (x.gas) { s2g += (rel * rel) * x.wgtc; swg += x.wgtc; }
                    else { s2s += (rel * rel) * x.wgtc; sws += x.wgtc; }
                }
                for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) {
                    if (do_mix) x.velgrad[i][j] = mix * x.velgrad[i][j] + (1.0 - mix) * x.velgradold[i][j];
                    else x.velgrad[i][j] = mix * x.velgrad[i][j];
                }
            }
            if (!kinematic_controlled) {
                double dls = sws > 0.0 ? std::sqrt(s2s / sws) : 0.0;
                double dlg = swg > 0.0 ? std::sqrt(s2g / swg) : 0.0;
                double dl = std::max(dls, dlg);
                mix = std::max(1.0e-8, std::min(1.0, 5.0e-2 / std::max(dl, 5.0e-2)));
            }
            solve_res();
            calc_velgradavg_corr();
            erre = erre / lvmavg;
            errs = errs / svmavg;
            errsbc = errsbc / svmavg;
            for (long v = 0; v < N; v++) copy3(vox[v].velgrad, vox[v].velgradold);
            if (pr.ictrl == 0) {
                M3 vs;
                sym33(velgradavg, vs);
                double evm = vm_strain(vs);
                pr.tdot = pr.devmapp / evm;
                pr.tdotref = pr.tdot;
            }
            if (errs <= pr.error && erre <= pr.error && errsbc <= pr.error) did_converge = true;
            if (pr.ictrl == -1) {
                if (pr.tdot > pr.tdotmin) {
                    double mv, mr, ms, md;
                    if (!did_converge && iter == pr.itmax) {
                        double tdot = pr.tdot;
                        int nsub = kinematic_substep(tdot, mv, mr, ms, md);
                        tdot = tdot / nsub;
                        tdot = std::max(pr.tdotmin, std::min(tdot, 0.5 * pr.tdot));
                        nsub = (int)std::ceil(pr.tdot / tdot);
                        if (nsub > 1) {
                            double remaining = std::max(0.0, proc_time_target - proc_time_done);
                            tdot_plan = tdot;
                            int nnew = (imicro - 1) + (int)std::ceil(remaining / tdot_plan);
                            total_macrosteps = total_macrosteps + nnew - pr.nsteps;
                            pr.nsteps = nnew;
                            pr.tdot = std::min(tdot_plan, remaining);
                            nconverged = 0;
                            iter = 0;
                            rollback();
                        }
                    } else if (did_converge) {
                        double tdot = pr.tdot;
                        int nsub = kinematic_substep(tdot, mv, mr, ms, md);
                        tdot = tdot / nsub;
                        if (md <= 1.0e-3) tdot = std::max(pr.tdotmin, std::min(tdot, 0.5 * pr.tdot));
                        else tdot = std::max(pr.tdotmin, tdot);
                        nsub = (int)std::ceil(pr.tdot / tdot);
                        if (nsub > 1) {
                            double remaining = std::max(0.0, proc_time_target - proc_time_done);
                            tdot_plan = tdot;
                            int nnew = (imicro - 1) + (int)std::ceil(remaining / tdot_plan);
                            total_macrosteps = total_macrosteps + nnew - pr.nsteps;
                            pr.nsteps = nnew;
                            pr.tdot = std::min(tdot_plan, remaining);
                            did_converge = false;
                            nconverged = 0;
                            iter = 0;
                            mix = 1.0;
                            rollback();
                        }
                    }
                } else if (iter == pr.itmax) {
                    accept_step = true;
                }
            }
            if (iter >= 100000) throw SolveError("equilibrium iteration did not converge", -4);
        }
        // accepted-step accumulation (LS-EVPFFT.f90:432-446)
        for (long v = 0; v < N; v++) {
            Voxel& x = vox[v];
            M3 vsym;
            for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) x.ept[i][j] = x.ept[i][j] + x.edotp[i][j] * pr.tdot;
            copy3(x.sg, x.sgt);
            sym33(x.velgrad, vsym);
            for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) x.disgradsym[i][j] = x.disgradsym[i][j] + vsym[i][j] * pr.tdot;
            x.epvm = x.epvm + vm_strain(x.edotp) * pr.tdot;
            double evm = vm_strain(vsym);
            if (evm > edotvmmx && !x.gas) edotvmmx = evm;
        }
        if (pr.iupdate == 1) {
            update_plastic_defgrad();
            update_grid_velgrad_node();
            update_defgrad();
            update_elastic_defgrad();
            update_el_stiff();
            update_tensor_config();
        }
        if (pr.iuphard == 1) update_hardening();
        // averages (LS-EVPFFT.f90:460-523)
        M3 vsym;
        sym33(velgradavg, vsym);
        lvmavg = vm_strain(velgradavg);
        dvmavg = vm_strain(vsym);
        evmavg = evmavg + dvmavg * pr.tdot;
        M3 ep = {}, ea = {}, el = {}, ed = {}, ss = {};
        double sum_gamma = 0, sum_g = 0, sum_gdot = 0, sum_ggdot = 0, nsolid = 0, nsys_solid = 0;
        for (long v = 0; v < N; v++) {
            const Voxel& x = vox[v];
            if (x.gas) continue;
            for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) {
                ep[i][j] = ep[i][j] + x.ept[i][j] * x.wgtc;
                ea[i][j] = ea[i][j] + x.disgradsym[i][j] * x.wgtc;
                el[i][j] = ea[i][j] + (x.disgradsym[i][j] - x.ept[i][j]) * x.wgtc;  // H4
                ed[i][j] = ed[i][j] + x.edotp[i][j] * x.wgtc;
                ss[i][j] = ss[i][j] + x.sgt[i][j] * x.wgtc;
            }
            sum_gamma = sum_gamma + x.gacumgr;
            nsolid = nsolid + 1.0;
            const Phase& ph = phase[x.phase - 1];
            for (int is = 0; is < ph.nsyst; is++) {
                double gs = 0.5 * (x.crss[is][0] + x.crss[is][1]);
                sum_g += gs;
                nsys_solid += 1.0;
                sum_gdot += std::fabs(x.gamdot[is]);
                sum_ggdot += std::fabs(x.gamdot[is]) * gs;
            }
        }
        for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) {
            epavg[i][j] = ep[i][j] / wphcsol; eavg[i][j] = ea[i][j] / wphcsol; eelavg[i][j] = el[i][j] / wphcsol;
            edotpavg[i][j] = ed[i][j] / wphcsol; sgsolavg[i][j] = ss[i][j] / wphcsol;
        }
        double gammaavg = nsolid > 0 ? sum_gamma / nsolid : 0.0;
        double gavg = nsys_solid > 0 ? sum_g / nsys_solid : 0.0;
        double geffavg = sum_gdot > 0 ? sum_ggdot / sum_gdot : gavg;
        evmpavg = vm_strain(epavg);
        dvmpavg = vm_strain(edotpavg);
        if (pr.iwfields == 1) {
            int aw = std::abs(pr.iwstep);
            bool w = (aw != 0 && imicro % aw == 0) || (pr.iwstep < 0 && imicro == pr.nsteps);
            if (w) write_vtk(imacroloop);
        }
        update_diagnostics();
        diag.erre = erre; diag.errs = errs; diag.errsbc = errsbc;
        diag.tdotref = pr.tdotref;
        diag.s33_target = pr.scauchy[2][2];
        diag.s33 = sgavg[2][2];
        diag.s33_sol = sgsolavg[2][2];
        double tdot_used = pr.tdot;
        if (pr.ictrl == -1) {
            proc_time_done = proc_time_done + tdot_used;
            pr.tdot = tdot_plan;
        }
        diag.devm_inc_max = edotvmmx * tdot_used;
        sim_time = sim_time + tdot_used;
        wall_time = (double)(std::time(nullptr) - start);
        write_rows(iter, imacroloop, ipr, sim_time, wall_time, tdot_used, diag.tdotref, gammaavg, gavg, geffavg);
        // ramp tdot back up (LS-EVPFFT.f90:557-581)
        if (pr.ictrl == -1) {
            if (tdot_plan < pr.tdotref && nconverged >= 5) {
                nconverged = 0;
                tdot_plan = std::min(2.0 * tdot_plan, pr.tdotref);
                double remaining = std::max(0.0, proc_time_target - proc_time_done);
                int left = (int)std::ceil(remaining / tdot_plan);
                int nnew = imicro + left;
                total_macrosteps = total_macrosteps + nnew - pr.nsteps;
                pr.nsteps = nnew;
                pr.tdot = (remaining > 0.0) ? std::min(tdot_plan, remaining) : tdot_plan;
            }
        } else if (pr.tdot < pr.tdotref && nconverged >= 5) {
            nconverged = 0;
            double tdot = pr.tdot;
            pr.tdot = std::min(2.0 * pr.tdot, pr.tdotref);
            int left = pr.nsteps - imicro;
            left = (int)std::ceil((double)left * tdot / pr.tdot);
            total_macrosteps = total_macrosteps + left - (pr.nsteps - imicro);
            pr.nsteps = imicro + left;
        }
        if (did_converge) nconverged++;
        calc_c0();
        imacroloop++;
        return true;
    }

    long get_field(const std::string& name, double* out, long n) const {
        auto need = [&](long per) { return per * N <= n; };
        auto put33 = [&](const M3 Voxel::*f) -> long {
            if (!need(9)) return -1;
            for (long v = 0; v < N; v++) for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) out[9 * v + 3 * i + j] = (vox[v].*f)[i][j];
            return 9 * N;
        };
        if (name == "sg") return put33(&Voxel::sg);
        if (name == "sgt") return put33(&Voxel::sgt);
        if (name == "velgrad") return put33(&Voxel::velgrad);
        if (name == "velgradold") return put33(&Voxel::velgradold);
        if (name == "defgrad") return put33(&Voxel::F);
        if (name == "defgradinv") return put33(&Voxel::Finv);
        if (name == "defgrade") return put33(&Voxel::Fe);
        if (name == "defgradp") return put33(&Voxel::Fp);
        if (name == "edotp") return put33(&Voxel::edotp);
        if (name == "ept") return put33(&Voxel::ept);
        if (name == "disgradsym") return put33(&Voxel::disgradsym);
        if (name == "dvelgradref") return put33(&Voxel::dvelgradref);
        int nsys = 0;
        for (auto& ph : phase) nsys = std::max(nsys, ph.nsyst);
        if (name == "gamdot") {
            if (!need(nsys)) return -1;
            for (long v = 0; v < N; v++) for (int s = 0; s < nsys; s++) out[nsys * v + s] = vox[v].gamdot[s];
            return nsys * N;
        }
        if (name == "crss" || name == "trialtau") {
            if (!need(2 * nsys)) return -1;
            for (long v = 0; v < N; v++) for (int s = 0; s < nsys; s++) for (int c = 0; c < 2; c++)
                out[2 * nsys * v + 2 * s + c] = (name == "crss") ? vox[v].crss[s][c] : vox[v].trialtau[s][c];
            return 2 * nsys * N;
        }
        if (name == "sch") {
            if (!need(5 * nsys)) return -1;
            for (long v = 0; v < N; v++) for (int s = 0; s < nsys; s++) for (int c = 0; c < 5; c++) out[5 * nsys * v + 5 * s + c] = vox[v].sch[s][c];
            return 5 * nsys * N;
        }
        if (name == "c066mod" || name == "sg66") {
            if (!need(36)) return -1;
            for (long v = 0; v < N; v++) for (int i = 0; i < 6; i++) for (int j = 0; j < 6; j++)
                out[36 * v + 6 * i + j] = (name == "c066mod") ? vox[v].c066mod[i][j] : vox[v].sg66[i][j];
            return 36 * N;
        }
        auto put1 = [&](double Voxel::*f) -> long {
            if (!need(1)) return -1;
            for (long v = 0; v < N; v++) out[v] = vox[v].*f;
            return N;
        };
        if (name == "detF") return put1(&Voxel::detF);
        if (name == "wgtc") return put1(&Voxel::wgtc);
        if (name == "gacumgr") return put1(&Voxel::gacumgr);
        if (name == "epvm") return put1(&Voxel::epvm);
        if (name == "macro") {  // c066, c0, s0, de_ds (reference-medium state)
            if (n < 279) return -1;
            std::memcpy(out, c066, sizeof(M6));
            std::memcpy(out + 36, c0, sizeof(T4));
            std::memcpy(out + 117, s0, sizeof(T4));
            std::memcpy(out + 198, de_ds, sizeof(T4));
            return 279;
        }
        if (name == "xnode") {
            long m = (long)xnode.size();
            if (m > n) return -1;
            std::memcpy(out, xnode.data(), sizeof(double) * m);
            return m;
        }
        return -1;
    }
};

void set_err(char* err, int errlen, const std::string& m) {
    if (err && errlen > 0) {
        std::strncpy(err, m.c_str(), errlen - 1);
        err[errlen - 1] = '\0';
    }
}

}  // namespace

struct oracle_solve {
    Oracle o;
};

extern "C" {

oracle_solve* oracle_open(const char* fft_in, const char* out_dir, int mix, int modal, int nthreads, int write_files, char* err,
                          int errlen) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    oracle_solve* s = new oracle_solve();
    s->o.write_files = (write_files != 0);
    s->o.verbose = (write_files == 2);
    try {
        s->o.open(fft_in, out_dir ? out_dir : "evpfft_outputs/", mix, modal);
    } catch (std::exception& e) {
        set_err(err, errlen, e.what());
        delete s;
        return nullptr;
    }
    return s;
}

int oracle_advance(oracle_solve* s, int nmacro) {
    int done = 0;
    try {
        for (int i = 0; i < nmacro; i++) {
            if (!s->o.macrostep()) break;
            done++;
        }
    } catch (SolveError& e) {
        std::fprintf(stderr, "oracle: %s\n", e.what());
        return e.code;
    } catch (std::exception& e) {
        std::fprintf(stderr, "oracle: %s\n", e.what());
        return -1;
    }
    return done;
}

long oracle_get_field(oracle_solve* s, const char* name, double* out, long n) { return s->o.get_field(name, out, n); }

int oracle_last_rows(oracle_solve* s, double* r51, double* d44) {
    if (r51) std::memcpy(r51, s->o.last_results, sizeof(s->o.last_results));
    if (d44) std::memcpy(d44, s->o.last_diag, sizeof(s->o.last_diag));
    return 0;
}

long oracle_total_iters(oracle_solve* s) { return s->o.total_iters; }

int oracle_grid(oracle_solve* s, int* n1, int* n2, int* n3) {
    *n1 = s->o.n1; *n2 = s->o.n2; *n3 = s->o.n3;
    return 0;
}

void oracle_close(oracle_solve* s) { delete s; }

int oracle_run(const char* fft_in, const char* out_dir, int mix, int modal, int nthreads, char* err, int errlen) {
    oracle_solve* s = oracle_open(fft_in, out_dir, mix, modal, nthreads, 1, err, errlen);
    if (!s) return -1;
    int rc = 0;
    while (true) {
        int d = oracle_advance(s, 1);
        if (d < 0) { rc = d; set_err(err, errlen, "solve failed"); break; }
        if (d == 0) break;
    }
    oracle_close(s);
    return rc;
}

void oracle_chg_basis_t2_to_b6(const double* c33, double* b6) {
    M3 c; std::memcpy(c, c33, sizeof(M3)); t2_to_b6(c, b6);
}
void oracle_chg_basis_b6_to_t2(const double* b6, double* c33) {
    M3 c; b6_to_t2(b6, c); std::memcpy(c33, c, sizeof(M3));
}
void oracle_chg_basis_t4_to_b66(const double* c3333, double* b66) {
    T4 c; M6 b; std::memcpy(c, c3333, sizeof(T4)); t4_to_b66(c, b); std::memcpy(b66, b, sizeof(M6));
}
void oracle_chg_basis_b66_to_t4(const double* b66, double* c3333) {
    T4 c; M6 b; std::memcpy(b, b66, sizeof(M6)); b66_to_t4(b, c); std::memcpy(c3333, c, sizeof(T4));
}
void oracle_expm_adaptive(const double* a33, double* e33) {
    M3 a, e; std::memcpy(a, a33, sizeof(M3)); expm_adaptive(a, e); std::memcpy(e33, e, sizeof(M3));
}
void oracle_polar(const double* f33, double* r33, double* u33) {
    M3 f, r, u; std::memcpy(f, f33, sizeof(M3)); polar(f, r, u); std::memcpy(r33, r, sizeof(M3)); std::memcpy(u33, u, sizeof(M3));
}
double oracle_cond1_6x6(const double* a66) {
    M6 a; std::memcpy(a, a66, sizeof(M6)); return cond1_est_6x6(a);
}
void oracle_fft3(double* data, int ncomp, int n1, int n2, int n3, int sign) {
    Fft1 p1, p2, p3;
    p1.init(n1, sign); p2.init(n2, sign); p3.init(n3, sign);
    cplx* c = reinterpret_cast<cplx*>(data);
    long N = (long)n1 * n2 * n3;
    for (int k = 0; k < ncomp; k++) fft3_field(c + k * N, n1, n2, n3, p1, p2, p3);
}
int oracle_green_apply(const double* tau9, double* out9, int n1, int n2, int n3, const double* c0, const double* s0) {
    // form_G (igamma=0) + convolution_with_Goper on a bare grid (various_functions.f90:640-809, 966-1059)
    try {
        Oracle o;
        o.n1 = n1; o.n2 = n2; o.n3 = n3;
        o.wgt = 1.0 / ((double)n1 * n2 * n3);
        o.init_micro();
        o.process.assign(1, Process());
        o.ipr = 1;
        std::memcpy(o.c0, c0, sizeof(T4));
        std::memcpy(o.s0, s0, sizeof(T4));
        o.form_G();
        const long N = o.N;
        for (long v = 0; v < N; v++)
            for (int c = 0; c < 9; c++) o.vox[v].sgPK1[c / 3][c % 3] = tau9[(long)c * N + v];
        o.convolution();
        for (long v = 0; v < N; v++)
            for (int c = 0; c < 9; c++) out9[(long)c * N + v] = o.vox[v].dvelgradref[c / 3][c % 3];
    } catch (std::exception& e) {
        std::fprintf(stderr, "oracle_green_apply: %s\n", e.what());
        return -1;
    }
    return 0;
}

// harden for one voxel of a one-mode phase: nsyst systems with Voce parameters tau1, thet0, thet1,
// the latent-hardening matrix hard (nsyst x nsyst, row-major), slip rates gamdot, accumulated shear
// gamma0 and committed resistances crss (nsyst x 2) over a step tdot; new resistances in tau_out.
double oracle_harden(int nsyst, double tau1, double thet0, double thet1, const double* hard, const double* gamdot,
                     double gamma0, const double* crss_nx2, double tdot, double* tau_out) {
    Phase ph;
    ph.nsyst = nsyst;
    ph.nmodes = 1;
    ph.nsm[0] = nsyst;
    for (int s = 0; s < nsyst; s++) {
        ph.tau[s][2] = tau1;
        ph.thet[s][0] = thet0;
        ph.thet[s][1] = thet1;
        for (int t = 0; t < nsyst; t++) ph.hard[s][t] = hard[nsyst * s + t];
    }
    double cr[NSYSMX][2], tau[NSYSMX][2], gamma1 = 0.0, gd[NSYSMX] = {};
    for (int s = 0; s < nsyst; s++) {
        cr[s][0] = crss_nx2[2 * s];
        cr[s][1] = crss_nx2[2 * s + 1];
        gd[s] = gamdot[s];
    }
    Oracle::harden_rates(ph, gd, gamma0, cr, tdot, tau, gamma1);
    for (int s = 0; s < nsyst; s++) {
        tau_out[2 * s] = tau[s][0];
        tau_out[2 * s + 1] = tau[s][1];
    }
    return gamma1;
}

void oracle_plastic_rate(const double* sch5xn, const double* trialtau_nx2, const double* nrs, const double* gamd0, int nsyst,
                         const double* sg6, double* edotp6, double* dedotp66, double* gamdot) {
    Phase ph;
    ph.nsyst = nsyst;
    double sch[NSYSMX][5], tt[NSYSMX][2];
    for (int s = 0; s < nsyst; s++) {
        ph.nrs[s] = nrs[s]; ph.gamd0[s] = gamd0[s];
        for (int c = 0; c < 5; c++) sch[s][c] = sch5xn[5 * s + c];
        tt[s][0] = trialtau_nx2[2 * s]; tt[s][1] = trialtau_nx2[2 * s + 1];
    }
    double d[6][6];
    Oracle::plastic_strain_rate(sg6, ph, sch, tt, gamdot, edotp6, d);
    std::memcpy(dedotp66, d, sizeof(d));
}

}  // extern "C"
