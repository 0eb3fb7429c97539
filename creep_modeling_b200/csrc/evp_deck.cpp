// evp_deck.cpp -- fft.in / cupl2.sx / cuel.sx / microstructure parser.
// Follows IO_functions.f90:6-812 (load_input, data_crystal, data_crystal_elast,
// data_grain) read by read, with Fortran list-directed record semantics.
#include "evp_deck.h"
#include "evp_math.cuh"

#include <algorithm>
#include <atomic>
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <thread>
#include <unistd.h>

namespace evp {
namespace {

// One microstructure record "phi1 Phi phi2 i j k grain phase" with blanks, tabs or
// commas between values: the common form without Fortran 'd' exponents.
bool micro_fast(const char* p, const char* e, double* e3, long* i5) {
    auto skip = [&]() {
        while (p < e && (*p == ' ' || *p == '\t' || *p == ',')) p++;
        if (p < e && *p == '+') p++;
    };
    for (int k = 0; k < 3; k++) {
        skip();
        auto r = std::from_chars(p, e, e3[k]);
        if (r.ec != std::errc() || (r.ptr < e && (*r.ptr == 'd' || *r.ptr == 'D'))) return false;
        p = r.ptr;
    }
    for (int k = 0; k < 5; k++) {
        skip();
        auto r = std::from_chars(p, e, i5[k]);
        if (r.ec != std::errc()) return false;
        p = r.ptr;
    }
    return true;
}
// The same record read the general way ('d' exponents allowed).
bool micro_slow(const char* p, const char* e, double* e3, long* i5) {
    std::string rec(p, e - p);
    for (char& c : rec)
        if (c == ',' || c == '\t') c = ' ';
        else if (c == 'd' || c == 'D') c = 'e';
    const char* s = rec.c_str();
    char* q = nullptr;
    for (int k = 0; k < 3; k++) {
        e3[k] = std::strtod(s, &q);
        if (q == s) return false;
        s = q;
    }
    for (int k = 0; k < 5; k++) {
        i5[k] = std::strtol(s, &q, 10);
        if (q == s) return false;
        s = q;
    }
    return true;
}

// A file as a list of records; list-directed reads consume whole records.
class Records {
public:
    explicit Records(const std::string& path) : path_(path) {
        FILE* f = std::fopen(path.c_str(), "rb");
        if (!f) throw DeckError("cannot open file '" + path + "'", -1);
        std::fseek(f, 0, SEEK_END);
        long n = std::ftell(f);
        std::fseek(f, 0, SEEK_SET);
        buf_.resize(n > 0 ? n : 0);
        if (n > 0 && std::fread(&buf_[0], 1, n, f) != (size_t)n) { std::fclose(f); throw DeckError("read error on '" + path + "'", -1); }
        std::fclose(f);
        size_t s = 0;
        for (size_t i = 0; i <= buf_.size(); i++) {
            if (i == buf_.size() || buf_[i] == '\n') {
                size_t e = i;
                if (e > s && buf_[e - 1] == '\r') e--;
                if (i < buf_.size() || e > s) { starts_.push_back(s); ends_.push_back(e); }
                s = i + 1;
            }
        }
    }
    // read(u,'(a)')
    std::string line() {
        check();
        std::string r = buf_.substr(starts_[pos_], ends_[pos_] - starts_[pos_]);
        pos_++;
        return r;
    }
    // read(u,*) with an empty list
    void skip() { check(); pos_++; }
    // read(u,*) of n items: returns tokens; continues over records; '/' ends the list
    std::vector<std::string> tokens(size_t n) {
        std::vector<std::string> out;
        while (out.size() < n) {
            check();
            const char* p = buf_.data() + starts_[pos_];
            const char* e = buf_.data() + ends_[pos_];
            pos_++;
            bool slash = false;
            while (p < e && out.size() < n) {
                char c = *p;
                if (c == ' ' || c == '\t' || c == ',') { p++; continue; }
                if (c == '/') { slash = true; break; }
                const char* q = p;
                while (q < e && *q != ' ' && *q != '\t' && *q != ',' && *q != '/') q++;
                out.emplace_back(p, q - p);
                p = q;
            }
            if (slash) break;
        }
        if (out.size() < n) throw DeckError("too few values in '" + path_ + "'", -1);
        return out;
    }
    double real(const std::string& t) const {
        std::string s = t;
        for (char& c : s)
            if (c == 'd' || c == 'D') c = 'e';
        char* end = nullptr;
        double v = std::strtod(s.c_str(), &end);
        if (end == s.c_str() || *end) throw DeckError("bad real '" + t + "' in '" + path_ + "'", -1);
        return v;
    }
    long integer(const std::string& t) const {
        char* end = nullptr;
        long v = std::strtol(t.c_str(), &end, 10);
        if (end == t.c_str() || *end) throw DeckError("bad integer '" + t + "' in '" + path_ + "'", -1);
        return v;
    }
    std::vector<double> reals(size_t n) { auto t = tokens(n); std::vector<double> v; for (auto& s : t) v.push_back(real(s)); return v; }
    std::vector<long> ints(size_t n) { auto t = tokens(n); std::vector<long> v; for (auto& s : t) v.push_back(integer(s)); return v; }
    // microstructure records (3 reals + 5 integers per line), records pos_ .. pos_ + n - 1,
    // parsed on several host threads into e3[3n], i5[5n]
    void micro_records(size_t n, double* e3, long* i5) {
        if (pos_ + n > starts_.size()) throw DeckError("unexpected end of file in '" + path_ + "'", -1);
        const size_t first = pos_;
        unsigned nt = std::thread::hardware_concurrency();
        nt = nt < 1 ? 1 : (nt > 16 ? 16 : nt);
        if (n < 4096) nt = 1;
        std::atomic<long long> bad{-1};
        auto work = [&](size_t a, size_t b) {
            for (size_t k = a; k < b; k++) {
                const char* p = buf_.data() + starts_[first + k];
                const char* e = buf_.data() + ends_[first + k];
                if (!micro_fast(p, e, e3 + 3 * k, i5 + 5 * k) && !micro_slow(p, e, e3 + 3 * k, i5 + 5 * k)) {
                    long long expect = -1;
                    bad.compare_exchange_strong(expect, (long long)k);
                    return;
                }
            }
        };
        if (nt == 1) {
            work(0, n);
        } else {
            std::vector<std::thread> th;
            const size_t chunk = (n + nt - 1) / nt;
            for (unsigned t = 0; t < nt; t++) {
                const size_t a = t * chunk, b = std::min(n, a + chunk);
                if (a < b) th.emplace_back(work, a, b);
            }
            for (auto& t : th) t.join();
        }
        if (bad.load() >= 0) throw DeckError("short microstructure record in '" + path_ + "'", -1);
        pos_ += n;
    }

private:
    void check() const {
        if (pos_ >= starts_.size()) throw DeckError("unexpected end of file in '" + path_ + "'", -1);
    }
    std::string path_, buf_;
    std::vector<size_t> starts_, ends_;
    size_t pos_ = 0;
};

std::string strip(const std::string& s) {
    size_t a = s.find_first_not_of(" \t");
    if (a == std::string::npos) return "";
    size_t b = s.find_last_not_of(" \t");
    return s.substr(a, b - a + 1);
}

// data_crystal (IO_functions.f90:367-638)
void read_slip_file(const std::string& path, PhaseData& ph) {
    Records r(path);
    r.line();
    std::string icryst = r.line().substr(0, 3);
    std::vector<double> cdim = r.reals(3);
    double covera = cdim[2] / cdim[0];
    int nmodesx = (int)r.ints(1)[0];
    int nmodes = (int)r.ints(1)[0];
    if (nmodes > kMaxModes) throw DeckError("nmodes exceeds nmodmx=3", -2);
    if (nmodesx > 10) throw DeckError("more than 10 modes listed", -2);
    std::vector<long> mode = r.ints(nmodes);
    ph.nmodes = nmodes;
    bool hex = (icryst == "HEX" || icryst == "TRI" || icryst == "hex" || icryst == "tri");
    bool cub = (icryst == "CUB" || icryst == "ORT" || icryst == "cub" || icryst == "ort");
    double hselfx[10] = {}, hlatex[10][10] = {};
    int nsyst = 0, kount = 1;
    for (int nm = 1; nm <= nmodesx; nm++) {
        r.line();
        auto t = r.tokens(6);
        int modex = (int)r.integer(t[0]), nsmx = (int)r.integer(t[1]);
        double nrsx = r.real(t[2]), gamd0x = r.real(t[3]), twshx = r.real(t[4]);
        auto h = r.reals(6);
        double tau0xf = h[0], tau0xb = h[1], tau1x = h[2], thet0x = h[3], thet1x = h[4], hpfacx = h[5];
        auto hl = r.reals(1 + nmodesx);
        hselfx[nm - 1] = hl[0];
        for (int j = 0; j < nmodesx; j++) hlatex[nm - 1][j] = hl[1 + j];
        if (kount > nmodes || modex != mode[kount - 1]) {
            for (int iz = 0; iz < nsmx; iz++) r.skip();
            continue;
        }
        if (thet0x < thet1x) throw DeckError("initial hardening lower than final hardening", -1);
        if (tau1x <= 1.e-6) { tau1x = 1.e-6; thet0x = thet1x; }
        hselfx[kount - 1] = hselfx[nm - 1];
        for (int i = 0; i < nmodes; i++) hlatex[kount - 1][i] = hlatex[nm - 1][mode[i] - 1];
        if (!hex && !cub) throw DeckError("cannot identify the crystal symmetry", -1);
        if (twshx > 1.0e-15) throw DeckError("twinning modes are not supported (ntwmmx = 0)", -2);
        ph.nsm[kount - 1] = nsmx;
        for (int js = 0; js < nsmx; js++) {
            auto v = r.ints(hex ? 8 : 6);
            if (++nsyst > kMaxSys) throw DeckError("nsyst exceeds nsysmx=24", -2);
            int s = nsyst - 1;
            ph.gamd0[s] = gamd0x; ph.nrs[s] = nrsx;
            ph.tau[s][0] = tau0xf; ph.tau[s][1] = tau0xb; ph.tau[s][2] = tau1x;
            ph.thet[s][0] = thet0x; ph.thet[s][1] = thet1x; ph.hpfac[s] = hpfacx;
            double sn[3], sb[3];
            if (hex) {
                sn[0] = (double)v[0];
                sn[1] = ((double)v[0] + 2. * (double)v[1]) / std::sqrt(3.);
                sn[2] = (double)v[3] / covera;
                sb[0] = 3. / 2. * (double)v[4];
                sb[1] = ((double)v[4] / 2. + (double)v[5]) * std::sqrt(3.);
                sb[2] = (double)v[7] * covera;
            } else {
                for (int m = 0; m < 3; m++) { sn[m] = (double)v[m] / cdim[m]; sb[m] = (double)v[3 + m] * cdim[m]; }
            }
            double snor = std::sqrt(sn[0] * sn[0] + sn[1] * sn[1] + sn[2] * sn[2]);
            double qnor = std::sqrt(sb[0] * sb[0] + sb[1] * sb[1] + sb[2] * sb[2]);
            double prod = 0.;
            for (int j = 0; j < 3; j++) {
                double n_ = sn[j] / snor, b_ = sb[j] / qnor;
                if (std::fabs(n_) < 1.e-03) n_ = 0.;
                if (std::fabs(b_) < 1.e-03) b_ = 0.;
                ph.dnca[s][j] = n_;
                ph.dbca[s][j] = b_;
                prod += n_ * b_;
            }
            if (prod >= 1.e-3) throw DeckError("slip system is not orthogonal", -1);
        }
        ph.nsyst = nsyst;
        kount++;
    }
    int i = 0;
    for (int im = 0; im < nmodes; im++)
        for (int is = 0; is < ph.nsm[im]; is++) {
            int j = 0;
            for (int jm = 0; jm < nmodes; jm++)
                for (int js = 0; js < ph.nsm[jm]; js++) ph.hard[i][j++] = hlatex[im][jm];
            ph.hard[i][i] = hselfx[im];
            i++;
        }
}

// data_crystal_elast (IO_functions.f90:640-720)
void read_elastic_file(const std::string& path, PhaseData& ph) {
    Records r(path);
    int iso = (int)r.ints(1)[0];
    if (iso == 0) {
        double c66[36];
        for (int i = 0; i < 6; i++) {
            auto v = r.reals(6);
            for (int j = 0; j < 6; j++) c66[6 * i + j] = v[j];
        }
        for (int i = 0; i < 6; i++)
            for (int j = 0; j < 6; j++) {
                int a = ijv_a(i), b = ijv_b(i), c = ijv_a(j), d = ijv_b(j);
                double x = c66[6 * i + j];
                ph.C[((a * 3 + b) * 3 + c) * 3 + d] = x;
                ph.C[((b * 3 + a) * 3 + c) * 3 + d] = x;
                ph.C[((a * 3 + b) * 3 + d) * 3 + c] = x;
                ph.C[((b * 3 + a) * 3 + d) * 3 + c] = x;
            }
    } else {
        auto v = r.reals(2);
        double young = v[0], tnu = v[1];
        double tmu = young / (2.0 * (1. + tnu));
        double tla = 2.0 * tmu * tnu / (1.0 - 2.0 * tnu);
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++)
                for (int k = 0; k < 3; k++)
                    for (int l = 0; l < 3; l++) {
                        double dij = (i == j), dkl = (k == l), dik = (i == k), djl = (j == l), dil = (i == l), djk = (j == k);
                        ph.C[((i * 3 + j) * 3 + k) * 3 + l] = tla * dij * dkl + 2.0 * tmu * ((dik * djl + dil * djk) / 2.0);
                    }
    }
}

}  // namespace

// Initial displacement file of IDISPINI (init_defgrad, IO_functions.f90:815-880): records
// "i j k u1 u2 u3" in loop order (the indices are read and ignored).  IDISPINI 1: one per cell
// centre, nodes by cell2node_tensor1 (various_functions.f90:2652-2691, x wrapped with n1);
// IDISPINI 2: one per node ((n1+1)(n2+1) x n3node), cells take their lower-corner node.
static void read_dispini(Deck& d, const std::string& path) {
    if (d.idispini != 1 && d.idispini != 2) throw DeckError("idispini must be 0, 1 or 2", -1);
    Records f(path);
    const int n1 = d.n1, n2 = d.n2, n3 = d.n3, nn3 = (n3 == 1) ? 1 : n3 + 1;
    const long long N = d.nvox();
    const long long nn1 = n1 + 1, nn2 = n2 + 1;
    auto node = [&](long long i, long long j, long long k) { return 3 * (i + nn1 * (j + nn2 * k)); };
    d.dispini.assign(3 * (size_t)N, 0.0);
    d.dispini_node.assign(3 * (size_t)(nn1 * nn2 * nn3), 0.0);
    if (d.idispini == 1) {
        for (long long v = 0; v < N; v++) {
            auto t = f.reals(6);
            for (int l = 0; l < 3; l++) d.dispini[3 * v + l] = t[3 + l];
        }
        auto cell = [&](long long i, long long j, long long k, int l) { return d.dispini[3 * (i + n1 * (j + (long long)n2 * k)) + l]; };
        for (long long k = 0; k < nn3; k++) {
            const long long k1 = (k + n3 - 1) % n3, k2 = k % n3;
            for (long long j = 0; j < nn2; j++) {
                const long long j1 = (j + n2 - 1) % n2, j2 = j % n2;
                for (long long i = 0; i < nn1; i++) {
                    const long long i1 = (i + n1 - 1) % n1, i2 = i % n1;
                    for (int l = 0; l < 3; l++)
                        d.dispini_node[node(i, j, k) + l] =
                            (cell(i2, j2, k2, l) + cell(i1, j2, k2, l) + cell(i2, j1, k2, l) + cell(i2, j2, k1, l) +
                             cell(i1, j1, k2, l) + cell(i1, j2, k1, l) + cell(i2, j1, k1, l) + cell(i1, j1, k1, l)) * 0.125;
                }
            }
        }
    } else {
        for (long long k = 0; k < nn3; k++)
            for (long long j = 0; j < nn2; j++)
                for (long long i = 0; i < nn1; i++) {
                    auto t = f.reals(6);
                    for (int l = 0; l < 3; l++) d.dispini_node[node(i, j, k) + l] = t[3 + l];
                }
        for (long long v = 0; v < N; v++) {
            const long long i = v % n1, j = (v / n1) % n2, k = v / ((long long)n1 * n2);
            for (int l = 0; l < 3; l++) d.dispini[3 * v + l] = d.dispini_node[node(i, j, k) + l];
        }
    }
}

Deck parse_deck(const std::string& fft_in) {
    Deck d;
    Records r(fft_in);
    d.nph = (int)r.ints(1)[0];
    auto g = r.ints(3);
    d.n1 = (int)g[0]; d.n2 = (int)g[1]; d.n3 = (int)g[2];
    if (d.n1 < 1 || d.n2 < 1 || d.n3 < 1) throw DeckError("grid dimensions must be positive", -1);
    if (d.nph < 1 || d.nph > kMaxPhases) throw DeckError("number of phases must be 1..3", -1);
    const long long N = d.nvox();
    d.wgt = 1.0 / (double)N;
    r.reals(3);  // delt: read, then forced to 4 (IO_functions.f90:62-66)
    const double voxel_vol = 4.0 * 4.0 * 4.0;
    r.line();
    std::string filetext = strip(r.line());
    d.phase.assign(d.nph, PhaseData());
    for (int iph = 0; iph < d.nph; iph++) {
        r.line();
        d.phase[iph].igas = (r.ints(1)[0] != 0);
        r.line();
        std::string fpl = strip(r.line());
        std::string fel = strip(r.line());
        if (!d.phase[iph].igas) {
            read_slip_file(fpl, d.phase[iph]);
            read_elastic_file(fel, d.phase[iph]);
        } else {
            d.has_gas = true;
        }
    }
    // data_grain (IO_functions.f90:722-812): voxel records in any order
    d.euler.assign(3 * N, 0.0);
    d.grain.assign(N, 0);
    d.phase_id.assign(N, 0);
    {
        Records m(filetext);
        std::vector<double> E3(3 * (size_t)N);
        std::vector<long> I5(5 * (size_t)N);
        m.micro_records((size_t)N, E3.data(), I5.data());
        for (long long kkk = 0; kkk < N; kkk++) {  // in file order: a later record for a voxel wins
            const double* e3 = &E3[3 * kkk];
            const long* i5 = &I5[5 * kkk];
            long ii = i5[0], jj = i5[1], kk = i5[2];
            if (ii < 1 || ii > d.n1 || jj < 1 || jj > d.n2 || kk < 1 || kk > d.n3)
                throw DeckError("voxel index out of range in microstructure file", -1);
            if (i5[4] < 1 || i5[4] > d.nph) throw DeckError("phase id out of range in microstructure file", -1);
            long long v = (ii - 1) + (long long)d.n1 * ((jj - 1) + (long long)d.n2 * (kk - 1));
            d.euler[3 * v] = e3[0]; d.euler[3 * v + 1] = e3[1]; d.euler[3 * v + 2] = e3[2];
            d.grain[v] = (int)i5[3];
            d.phase_id[v] = (int)i5[4];
        }
    }
    // Hall-Petch grain sizes (IO_functions.f90:107-138); the 1000-grain cap is lifted
    const double hp_kgr_default = 632 / 2.5;
    const double grain_dmin = 3.0 * std::pow(voxel_vol, 1.0 / 3.0);
    std::vector<std::vector<long long>> cnt(d.nph);
    for (long long v = 0; v < N; v++) {
        int p = d.phase_id[v] - 1;
        if (d.phase[p].igas) continue;
        int gid = d.grain[v];
        if (gid < 1) throw DeckError("grain id out of bounds for Hall-Petch init", -1);
        if ((long long)cnt[p].size() <= gid) cnt[p].resize(gid + 1, 0);
        cnt[p][gid]++;
    }
    d.hp_shift.assign(N, 0.0);
    for (long long v = 0; v < N; v++) {
        int p = d.phase_id[v] - 1;
        if (d.phase[p].igas) continue;
        long long nv = cnt[p][d.grain[v]];
        double gd = nv > 0 ? std::pow((double)nv * voxel_vol, 1.0 / 3.0) : 0.0;
        if (gd > 0.0) d.hp_shift[v] = hp_kgr_default / std::sqrt(std::max(gd, grain_dmin));
    }
    r.line();
    d.imicrosave = (int)r.ints(2)[1];
    d.complgas = r.reals(1)[0];
    r.line();
    d.idispini = (int)r.ints(1)[0];
    if (d.idispini > 0) read_dispini(d, strip(r.line()));
    d.nproc = (int)r.ints(1)[0];
    if (d.nproc < 1) throw DeckError("cannot have less than one processes", -1);
    d.process.assign(d.nproc, ProcessData());
    std::vector<double> eth_tab;  // 9 per grain id
    bool any_thermo = false;
    for (int ip = 0; ip < d.nproc; ip++) {
        ProcessData& p = d.process[ip];
        r.line(); r.line();
        for (int i = 0; i < 3; i++) { auto v = r.ints(3); for (int j = 0; j < 3; j++) p.iudot[3 * i + j] = (int)v[j]; }
        if (p.iudot[0] + p.iudot[4] + p.iudot[8] == 2) throw DeckError("check diagonal boundary conditions iudot", -1);
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++)
                if (i != j && p.iudot[3 * i + j] + p.iudot[3 * j + i] == 0) throw DeckError("check off-diagonal boundary conditions iudot", -1);
        r.skip();
        for (int i = 0; i < 3; i++) { auto v = r.reals(3); for (int j = 0; j < 3; j++) p.udot[3 * i + j] = v[j]; }
        sym33(p.udot, p.dsim);
        antisym33(p.udot, p.tomtot);
        p.dvm = vm_strain(p.dsim);
        for (int i = 0; i < 3; i++) p.idsim[i] = p.iudot[4 * i];
        p.idsim[3] = (p.iudot[5] == 1 && p.iudot[7] == 1);
        p.idsim[4] = (p.iudot[2] == 1 && p.iudot[6] == 1);
        p.idsim[5] = (p.iudot[1] == 1 && p.iudot[3] == 1);
        r.skip();
        { auto v = r.ints(3); p.iscau[0] = (int)v[0]; p.iscau[5] = (int)v[1]; p.iscau[4] = (int)v[2]; }
        { auto v = r.ints(2); p.iscau[1] = (int)v[0]; p.iscau[3] = (int)v[1]; }
        p.iscau[2] = (int)r.ints(1)[0];
        for (int i = 0; i < 6; i++)
            if (p.iscau[i] * p.idsim[i] != 0 || p.iscau[i] + p.idsim[i] != 1)
                throw DeckError("check boundary condits on strain-rate and stress", -1);
        r.skip();
        { auto v = r.reals(3); p.scauchy[0] = v[0]; p.scauchy[1] = v[1]; p.scauchy[2] = v[2]; }
        { auto v = r.reals(2); p.scauchy[4] = v[0]; p.scauchy[5] = v[1]; }
        p.scauchy[8] = r.reals(1)[0];
        p.scauchy[7] = p.scauchy[5]; p.scauchy[6] = p.scauchy[2]; p.scauchy[3] = p.scauchy[1];
        r.skip();
        { auto v = r.reals(4); p.tdot = v[0]; p.tdotref = v[1]; p.tdotmin = v[2]; p.devmmx = v[3]; }
        p.ictrl = (int)r.ints(1)[0];
        if (p.ictrl == 0) {
            p.devmapp = p.tdot;
            p.tdot = p.tdot / p.dvm;
            p.tdotref = p.tdot;
        } else if (p.ictrl > 0) {
            throw DeckError("ictrl>0 not implemented", -2);
        }
        r.skip();
        p.nsteps = (int)r.ints(1)[0];
        { auto v = r.reals(2); p.error = v[0]; p.erroral = v[1]; }
        p.itmax = (int)r.ints(1)[0];
        p.irecover = (int)r.ints(1)[0];
        if (p.irecover == 1 && ::access("stress.in", R_OK) != 0) throw DeckError("stress.in not found (IRECOVER=1)", -1);
        p.isave = (int)r.ints(1)[0];
        p.iupdate = (int)r.ints(1)[0];
        p.iuphard = (int)r.ints(1)[0];
        p.iwtex = (int)r.ints(1)[0];
        { auto v = r.ints(2); p.iwfields = (int)v[0]; p.iwstep = (int)v[1]; }
        { auto t = r.tokens(2); p.xc0 = r.real(t[0]); p.igamma = (int)r.integer(t[1]); }
        if (!(p.nsteps > 0)) throw DeckError("nsteps must be positive", -1);
        if (!(p.error > 0 || p.erroral > 0)) throw DeckError("error and erroral tolerances must be positive", -1);
        if (!(p.itmax > 0)) throw DeckError("itmax must be positive", -1);
        if (!(p.irecover == 0 || p.irecover == 1)) throw DeckError("irecover must be 0 or 1", -1);
        if (!(p.isave == 0 || p.isave == 1)) throw DeckError("isave must be 0 or 1", -1);
        if (!(p.iupdate == 0 || p.iupdate == 1)) throw DeckError("iupdate must be 0 or 1", -1);
        if (!(p.iuphard == 0 || p.iuphard == 1)) throw DeckError("iuphard must be 0 or 1", -1);
        if (!(p.iwtex == 0 || p.iwtex == 1)) throw DeckError("iwtex must be 0 or 1", -1);
        if (!(p.iwfields == 0 || p.iwfields == 1)) throw DeckError("iwfields must be 0 or 1", -1);
        if (!(p.igamma == 0 || p.igamma == 1 || p.igamma == 2)) throw DeckError("igamma must be 0, 1 or 2", -1);
        p.ithermo = (int)r.ints(1)[0];
        if (p.ithermo == 1) {
            any_thermo = true;
            Records th(strip(r.line()));
            long ngr = th.ints(1)[0];
            if ((long)eth_tab.size() < 9 * (ngr + 1)) eth_tab.resize(9 * (ngr + 1), 0.0);
            for (long ig = 1; ig <= ngr; ig++) {
                auto v = th.reals(6);
                double* e = &eth_tab[9 * ig];
                e[0] = v[0]; e[4] = v[1]; e[8] = v[2]; e[5] = v[3]; e[6] = v[4]; e[1] = v[5];
                e[7] = e[5]; e[2] = e[6]; e[3] = e[1];
            }
        }
    }
    if (any_thermo) {
        d.eth.assign(9 * N, 0.0);
        for (long long v = 0; v < N; v++) {
            long gid = d.grain[v];
            if (gid >= 1 && 9 * (gid + 1) <= (long)eth_tab.size())
                for (int c = 0; c < 9; c++) d.eth[9 * v + c] = eth_tab[9 * gid + c];
        }
    }
    return d;
}

}  // namespace evp
