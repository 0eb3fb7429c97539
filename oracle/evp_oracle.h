/*
 * evp_oracle.h -- C API of the CPU FP64 oracle for the LS-EVPFFT solve.
 *
 * TEST INFRASTRUCTURE ONLY.  The oracle is a plain-C++ restatement of the
 * reference Fortran solver (gdebrun2/creep_modeling, lsevpfft/src/ Fortran sources).  It is
 * the checker for the CUDA product and the timed CPU baseline; the product
 * never links, loads or calls it.
 *
 * Parity status: UNPINNED against the Fortran executable itself (no Fortran
 * compiler, FFTW or LAPACK exists where this was written, and the reference
 * ships no golden outputs).  The oracle is pinned instead by analytic
 * known-answer tests and by numpy/scipy golden vectors (tests/golden/).
 */
#ifndef EVP_ORACLE_H
#define EVP_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_solve oracle_solve;

/* Parse the deck (fft.in grammar of IO_functions.f90:6-365), initialise the
 * state exactly as LS-EVPFFT.f90:144-178 does.  write_files != 0 writes
 * results.csv / diagnostics.csv / VTK into out_dir like the executable.
 * Returns NULL on error (message in err). */
oracle_solve* oracle_open(const char* fft_in, const char* out_dir, int mix,
                          int modal, int nthreads, int write_files,
                          char* err, int errlen);

/* Advance up to nmacro macrosteps (LS-EVPFFT.f90:198-589).  Returns the
 * number of macrosteps done (0 once the whole deck is finished), or a
 * negative status on failure. */
int oracle_advance(oracle_solve* s, int nmacro);

/* Copy a per-voxel field (voxel index v = i + n1*(j + n2*k), components
 * innermost; 3x3 tensors in (row, col) order) into out.  Returns the number
 * of doubles written, or -1 for an unknown name / short buffer. */
long oracle_get_field(oracle_solve* s, const char* name, double* out, long n);

/* Last results.csv row (53 numbers, column order of IO_functions.f90:1264-1271)
 * and diagnostics.csv row (44 numbers, types.f90:787-798). */
int oracle_last_rows(oracle_solve* s, double* results53, double* diag44);

/* Sum of global equilibrium iterations executed so far, and macrosteps. */
long oracle_total_iters(oracle_solve* s);
int oracle_grid(oracle_solve* s, int* n1, int* n2, int* n3);
void oracle_close(oracle_solve* s);

/* Whole-run entry point with the executable's semantics. 0 = ok. */
int oracle_run(const char* fft_in, const char* out_dir, int mix, int modal,
               int nthreads, char* err, int errlen);

/* ---- unit-level entry points used by the known-answer tests ---- */
void oracle_chg_basis_t2_to_b6(const double* c33, double* b6);
void oracle_chg_basis_b6_to_t2(const double* b6, double* c33);
void oracle_chg_basis_t4_to_b66(const double* c3333, double* b66);
void oracle_chg_basis_b66_to_t4(const double* b66, double* c3333);
void oracle_expm_adaptive(const double* a33, double* e33);
void oracle_polar(const double* f33, double* r33, double* u33);
double oracle_cond1_6x6(const double* a66);
/* In-place 3-D DFT of ncomp complex fields (interleaved re,im), x fastest.
 * sign = -1 forward, +1 backward (unnormalised). */
void oracle_fft3(double* data, int ncomp, int n1, int n2, int n3, int sign);
/* Green operator (igamma=0) applied to 9 real fields tau9[c*N + v]. 0 = ok. */
int oracle_green_apply(const double* tau9, double* out9, int n1, int n2, int n3, const double* c0, const double* s0);
/* One constitutive evaluation (plastic_strain_rate + elastic_strain_rate). */
void oracle_plastic_rate(const double* sch5xn, const double* trialtau_nx2,
                         const double* nrs, const double* gamd0, int nsyst,
                         const double* sg6, double* edotp6, double* dedotp66,
                         double* gamdot);
/* harden (various_functions.f90:1439-1491) for one voxel of a one-mode phase: new resistances
 * (nsyst x 2) in tau_out; returns the new accumulated shear. */
double oracle_harden(int nsyst, double tau1, double thet0, double thet1, const double* hard,
                     const double* gamdot, double gamma0, const double* crss_nx2, double tdot,
                     double* tau_out);

#ifdef __cplusplus
}
#endif
#endif
