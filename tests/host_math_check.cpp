// Host build of the device math helpers (evp_math.cuh compiles as plain C++), for CPU tests of
// identities the kernels rely on: the column-by-column inverse from LU factors gives the bits of
// the full [A | I] elimination, and the b-basis rotation Q c Q^T equals the index-by-index
// rotation of a fourth-order tensor followed by chg_basis.
#include "../creep_modeling_b200/csrc/evp_math.cuh"

#include <cstdint>
#include <cstring>
#include <random>

using namespace evp;

extern "C" {

// Number of 6x6 test matrices (random, some needing row interchanges) whose inverse by
// lu_unrolled + lu_inverse_column differs in any bit from inv_unrolled's.
int check_inverse_columns(int ntrials, unsigned seed) {
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<double> u(-1.0, 1.0);
    int bad = 0;
    for (int t = 0; t < ntrials; t++) {
        double a[36];
        for (int c = 0; c < 36; c++) a[c] = u(rng);
        if (t % 2 == 0)  // diagonally dominant half: no interchanges; the other half pivots
            for (int i = 0; i < 6; i++) a[7 * i] += 8.0;
        double full[36];
        std::memcpy(full, a, sizeof(full));
        const int info1 = inv_unrolled<6>(full);
        double J[36];
        int piv[6];
        std::memcpy(J, a, sizeof(J));
        const int info2 = lu_unrolled<6>(J, piv);
        double cols[36];
        for (int j = 0; j < 6; j++) {
            double x[6];
            lu_inverse_column<6>(J, piv, j, x);
            for (int i = 0; i < 6; i++) cols[6 * i + j] = x[i];
        }
        if (info1 != info2 || std::memcmp(full, cols, sizeof(full)) != 0) bad++;
    }
    return bad;
}

// Largest relative difference, over random minor- and major-symmetric stiffnesses c and random
// (non-orthogonal) maps a, between rot_b66(a) c66 rot_b66(a)^T and chg_basis of the rotation
// c'_ijkl = a_ip a_jq a_kr a_ls c_pqrs done index by index.
double check_rot_b66(int ntrials, unsigned seed) {
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<double> u(-1.0, 1.0);
    double worst = 0.0;
    for (int t = 0; t < ntrials; t++) {
        double X[36], c66[36], c4[81], a[9];
        for (int c = 0; c < 36; c++) X[c] = u(rng);
        for (int i = 0; i < 6; i++)  // c66 = X X^T: symmetric
            for (int j = 0; j < 6; j++) {
                double s = 0.0;
                for (int k = 0; k < 6; k++) s += X[6 * i + k] * X[6 * j + k];
                c66[6 * i + j] = s;
            }
        b66_to_t4(c66, c4);
        for (int c = 0; c < 9; c++) a[c] = u(rng) + ((c % 4 == 0) ? 2.0 : 0.0);
        double r4[81], ref[36];
        rotate4(a, c4, r4);
        t4_to_b66(r4, ref);
        double Q[36], QC[36], out[36];
        rot_b66(a, Q);
        for (int i = 0; i < 6; i++)
            for (int j = 0; j < 6; j++) {
                double s = 0.0;
                for (int k = 0; k < 6; k++) s += Q[6 * i + k] * c66[6 * k + j];
                QC[6 * i + j] = s;
            }
        double scale = 0.0;
        for (int c = 0; c < 36; c++) scale = std::fmax(scale, std::fabs(ref[c]));
        for (int i = 0; i < 6; i++)
            for (int j = 0; j < 6; j++) {
                double s = 0.0;
                for (int k = 0; k < 6; k++) s += QC[6 * i + k] * Q[6 * j + k];
                out[6 * i + j] = s;
                worst = std::fmax(worst, std::fabs(s - ref[6 * i + j]) / scale);
            }
    }
    return worst;
}

}  // extern "C"
