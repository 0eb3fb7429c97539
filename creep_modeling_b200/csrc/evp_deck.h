// evp_deck.h -- host-side model of the LS-EVPFFT input deck.
//
// Parses fft.in, the slip file (cupl2.sx), the elastic file (cuel.sx) and the
// microstructure .dat with the record semantics of the reference's Fortran
// list-directed READs (lsevpfft/src/IO_functions.f90:6-812).
#pragma once
#include <string>
#include <vector>
#include <stdexcept>

namespace evp {

constexpr int kMaxSys = 24;   // nsysmx (global.f90:16)
constexpr int kMaxModes = 3;  // nmodmx (global.f90:15)
constexpr int kMaxPhases = 3; // nphmx (global.f90:14)

struct DeckError : std::runtime_error {
    int code;
    DeckError(const std::string& m, int c = -1) : std::runtime_error(m), code(c) {}
};

// phase_type (types.f90:96-118), the fields the solve reads
struct PhaseData {
    bool igas = false;
    int nsyst = 0, nmodes = 0, nsm[kMaxModes] = {0, 0, 0};
    double nrs[kMaxSys] = {}, gamd0[kMaxSys] = {}, hpfac[kMaxSys] = {};
    double tau[kMaxSys][3] = {}, thet[kMaxSys][2] = {};
    double hard[kMaxSys][kMaxSys] = {};
    double dnca[kMaxSys][3] = {}, dbca[kMaxSys][3] = {};
    double C[81] = {};  // crystal stiffness (i,j,k,l)
};

// process_type (types.f90:120-152)
struct ProcessData {
    int ithermo = 0, iudot[9] = {}, idsim[6] = {}, iscau[6] = {}, ictrl = 0, nsteps = 0, itmax = 0;
    int irecover = 0, isave = 0, iupdate = 0, iuphard = 0, iwtex = 0, iwfields = 0, iwstep = 0, igamma = 0;
    double udot[9] = {}, dsim[9] = {}, tomtot[9] = {}, scauchy[9] = {};
    double dvm = 0, tdot = 0, tdotref = 0, tdotmin = 0, devmmx = 0, error = 0, erroral = 0, xc0 = 0, devmapp = 0;
};

struct Deck {
    int n1 = 0, n2 = 0, n3 = 0, nph = 0, nproc = 0, idispini = 0, imicrosave = 0;
    double wgt = 0.0, complgas = 0.0;
    std::vector<PhaseData> phase;
    std::vector<ProcessData> process;
    // per voxel, index v = i + n1*(j + n2*k)
    std::vector<double> euler;     // 3 per voxel, degrees (phi1, Phi, phi2)
    std::vector<int> grain, phase_id;
    std::vector<double> hp_shift;  // Hall-Petch tau0 shift per voxel (IO_functions.f90:107-199)
    std::vector<double> eth;       // 9 per voxel (only when some process has ithermo=1)
    // IDISPINI 1, 2 (IO_functions.f90:815-936): initial displacement at the cell centres (3 per voxel)
    // and at the nodes (3 per node, node index i + (n1+1)(j + (n2+1) k), k < n3node)
    std::vector<double> dispini, dispini_node;
    bool has_gas = false;
    long long nvox() const { return (long long)n1 * n2 * n3; }
};

// Parse a deck; relative file names inside fft.in resolve against the current
// working directory, as the reference's OPEN statements do.
Deck parse_deck(const std::string& fft_in);

}  // namespace evp
