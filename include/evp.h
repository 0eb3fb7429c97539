/*
 * evp.h -- C ABI of the B200-native LS-EVPFFT solver (libevp_b200.so).
 *
 * The reference solver is the Fortran executable lsevpfft/LS-EVPFFT, launched
 * as a separate process by utils/run.py:169-196 (run_solver) with
 *     LS-EVPFFT --nthreads n --in fft.in --out DIR --fftw_save P --mix m --modal a
 * (flag parsing at lsevpfft/src/LS-EVPFFT.f90:87-142) and talking to its
 * callers only through files: results.csv (IO_functions.f90:1237-1303),
 * diagnostics.csv (types.f90:760-834) and VTK (IO_functions.f90:945-1235).
 * These entry points replace that process.  Plain C types only; the library
 * owns every device allocation; strings are copied.
 *
 * Status codes: 0 ok; -1 deck or input-file error; -2 deck feature not
 * supported by this build; -3 singular matrix (the reference's `stop 1` in
 * lu_inverse / lu_eqsystem / dgesvd); -4 non-convergence or non-finite
 * state; -5 output-file error; -6 CUDA error or no device; -7 bad argument;
 * -8 the solve's wall-clock deadline passed (evp_set_deadline, evp_submit_deadline).
 */
#ifndef EVP_B200_H
#define EVP_B200_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct evp_solve evp_solve;

/* Caller-owned summary of one solve. */
typedef struct evp_report {
    int status;                  /* final status code */
    int macrosteps;              /* macrosteps completed */
    long long equilibrium_iters; /* sum of global equilibrium iterations executed (the `iter` column) */
    long long voxel_iters;       /* equilibrium_iters * number of voxels */
    double wall_s;               /* host wall time of the solve, seconds */
    double gpu_s;                /* device time of the macrostep loop (CUDA events), seconds */
    int n1, n2, n3;              /* grid */
    long long h2d_bytes;         /* host-to-device bytes copied so far (deck upload, per-step constants) */
    long long d2h_bytes;         /* device-to-host bytes copied so far (per-iteration sums, fields) */
} evp_report;

/* Flags for evp_open. */
#define EVP_WRITE_FILES 1  /* write results.csv, diagnostics.csv and VTK like the executable */
#define EVP_VERBOSE 2      /* print the progress line (various_functions.f90:2693-2743) */
#define EVP_WRITE_CSV 4    /* write results.csv and diagnostics.csv only (no VTK) */
#define EVP_PROFILE 8      /* time every kernel launch with CUDA events (evp_kernel_times) */
#define EVP_MIXED 16       /* mixed precision: the equilibrium iteration's spectrum, FFTs and Green-operator
                              application in FP32; local Newton, reductions and F/rotation updates in FP64 */

/* Whole solve with the executable's semantics: replaces one
 * `LS-EVPFFT --in fft_in --out out_dir --mix mix --modal modal` process
 * (LS-EVPFFT.f90:87-595).  nthreads is accepted for the same command line and
 * ignored.  fftw_save, the reference's FFTW wisdom file (fourier_functions.f90:35-66),
 * names the tile cache of the FFT passes here (evp_tune_cache); NULL or "": none. */
int evp_solve_file(const char* fft_in, const char* out_dir, int nthreads, const char* fftw_save, int mix, int modal,
                   evp_report* report);

/* Tile cache of the spectral passes for every later open in this process (the
 * counterpart of FFTW's wisdom file; path NULL or "": none).  Opening a solve whose
 * grid this process has not seen times the candidate tiles of the x-forward, y and
 * z-with-Green-operator passes on the device (a few milliseconds) unless the cache
 * file has them; the fastest are kept for the process and appended to the file, so
 * later processes read them.  The tile changes no result.  Its directory is created. */
int evp_tune_cache(const char* path);

/* Step-wise form of the same solve, for tests and the serving loop.
 * evp_open = load_input + initial_guess + start-up c0 (LS-EVPFFT.f90:144-178);
 * evp_advance runs up to nmacro macrosteps of LS-EVPFFT.f90:198-589 and
 * reports how many ran in *done (0 once the deck is finished). */
int evp_open(const char* fft_in, const char* out_dir, int mix, int modal, int flags, evp_solve** out);
int evp_advance(evp_solve* s, int nmacro, int* done);

/* Copy a per-voxel field to host memory (voxel v = i + n1*(j + n2*k),
 * components innermost, 3x3 tensors row-major).  Names: sg, sgt, velgrad,
 * velgradold, defgrad, defgradinv, defgrade, defgradp, edotp, ept,
 * disgradsym, dvelgradref, gamdot, crss, trialtau, sch, c066mod, sg66, detF,
 * wgtc, gacumgr, epvm, xnode.  *written = number of doubles copied. */
int evp_get_field(evp_solve* s, const char* name, double* host_out, long long capacity, long long* written);

/* Last results.csv row (51 values, IO_functions.f90:1264-1271 order) and
 * diagnostics.csv row (44 values, types.f90:787-798 order). */
int evp_last_rows(evp_solve* s, double* results51, double* diag44);
int evp_stats(evp_solve* s, evp_report* out);
/* Wall-clock budget for the rest of the solve, in seconds from now (<= 0: none).  The
 * solve checks it before every equilibrium iteration and, once it has passed, ends
 * with -8; the files written so far stay.  The reference has no counterpart (its
 * callers can only kill the process). */
int evp_set_deadline(evp_solve* s, double seconds);
int evp_close(evp_solve* s);

/* Per-kernel device time under EVP_PROFILE: fills up to cap entries of
 * names (each a NUL-terminated string of at most 31 chars, stored in
 * names[32*i]), launches and milliseconds; returns the number of kernels. */
int evp_kernel_times(evp_solve* s, char* names, long long* launches, double* ms, int cap);
/* Number of kernels this solve has launched so far (with or without EVP_PROFILE); -1 for a null handle. */
long long evp_kernel_launches(evp_solve* s);
/* Activity counters of the local Newton kernel since open (EVP_PROFILE solves only; no
 * counterpart in the reference): out6[0] warp passes of the evaluation loop, [1] voxel
 * evaluations done in those passes (five voxel groups per warp), [2] Newton steps, [3]
 * hardening updates, [4] voxels solved, [5] warp passes of the Newton-step loop.
 * [1] / (5 [0]) is the fraction of voxel slots that did useful work. */
int evp_newton_stats(evp_solve* s, long long* out6);

/* Operator-level entry: applies the periodic Green operator of a homogeneous
 * reference medium to a polarization field, the inner operator of every
 * equilibrium iteration (convolution_with_Goper with form_G igamma = 0,
 * lsevpfft/src/various_functions.f90:640-809 and 966-1059).
 * d_tau, d_out: caller-owned device arrays of 9 x N doubles, component c = 3*i+j
 * outermost (field[c*N + v], v = i + n1*(j + n2*k)); d_out may not alias d_tau.
 * c0, s0: host arrays of 81 doubles, the reference stiffness and its
 * compliance (4th-order, index ((i*3+j)*3+k)*3+l).  stream: a cudaStream_t or
 * NULL.  The scratch spectrum is allocated and freed inside the call. */
int evp_green_apply(const double* d_tau, double* d_out, int n1, int n2, int n3, const double* c0, const double* s0,
                    void* stream);

/* Allocation-free variant of evp_green_apply (no counterpart in the reference,
 * whose Fortran solver has no device and no allocator to avoid).  For callers
 * that cannot call cudaMalloc: their device memory belongs to another
 * allocator (a pre-reserved pool such as PyTorch's caching allocator, or a
 * serving loop whose HBM budget is already handed out), or they run
 * latency-critical loops that cannot take the device-wide synchronization of
 * cudaMalloc / cudaFree.  Same arguments and results as evp_green_apply; the
 * scratch lives in a fixed array of about 2.5 MB that every GPU loading this
 * library keeps until the process exits.  Limits: (n1/2+1)*n2*n3 <= 17408
 * (a 32^3 grid) and every edge <= 256; larger grids return -7 with a message.
 * The first call on a device resolves the array's address and should come
 * before any stream capture.  All calls on a device share the array, so calls
 * whose device work overlaps race and must be serialized by the caller. */
int evp_green_apply_noalloc(const double* d_tau, double* d_out, int n1, int n2, int n3, const double* c0,
                            const double* s0, void* stream);

/* ---- Batching: many solves advanced together (no counterpart in the reference, whose
 * callers run one solver process per solve and two or three at once, utils/run.py:169-196,
 * calibrate.py:1053-1057).
 *
 * Every equilibrium iteration of the batch is one launch per pass (stress average, the
 * five FFT passes with the Green operator, correction, local Newton; per kernel variant
 * and per 40 members) over all running members, whatever their grid sizes and material
 * parameters, followed by a device-side controller that does each member's serial tail
 * (averages, boundary-condition update, error norms, convergence and time-step rules)
 * without the host; those launches are captured once in a CUDA graph and replayed.
 * Members advance independently: one that converges writes its rows and starts its next
 * increment while the others keep iterating; one that fails stops with its status and
 * the others go on.  Each member's results are the same as when it runs alone. */
typedef struct evp_batch evp_batch;
int evp_batch_open(evp_batch** out);
/* Add a solve (same deck, flags and files as evp_open; EVP_PROFILE is ignored).  *slot
 * identifies it.  A deck or start-up error returns its status code (the slot, if
 * any, is then finished with that status). */
int evp_batch_add(evp_batch* b, const char* fft_in, const char* out_dir, int mix, int modal, int flags, int* slot);
/* Advance the running members by `rounds` rounds of a few iterations each; *running gets the
 * number of members still running. */
int evp_batch_step(evp_batch* b, int rounds, int* running);
/* *state: 0 running, 1 finished; rep->status is the member's status code once finished;
 * msg (msgcap bytes, may be NULL) its error message. */
int evp_batch_status(evp_batch* b, int slot, int* state, evp_report* rep, char* msg, int msgcap);
int evp_batch_close(evp_batch* b);
/* Run n decks as one batch to the end (the batched form of n evp_solve_file calls); reports[i]
 * describes deck i; returns 0 or the first nonzero status.  flags 0: EVP_WRITE_FILES. */
int evp_solve_files(int n, const char* const* fft_in, const char* const* out_dir, int mix, int modal, int flags,
                    evp_report* reports);

/* ---- Serving: a resident request loop (the reference has no counterpart; it
 * runs one solver process per request, utils/run.py:169-196, and calibrate.py
 * runs two or three such processes at once, calibrate.py:1053-1057).
 *
 * A server keeps every admitted solve's fields on the device until the solve
 * ends and writes the same files as evp_solve_file.  evp_submit reads the deck
 * on the caller's thread (a deck error makes the request done at once with its
 * status); requests then queue.  One engine thread runs the admitted solves as
 * batches (the evp_batch_* form: every equilibrium iteration is one launch per
 * pass over all of a batch's solves, whatever their grid sizes).  Between rounds of a few
 * iterations it admits queued requests, the one with the least work (voxels x
 * increments) first, while fewer than max_inflight solves run and the request's
 * estimated device footprint fits the budget beside the running ones; a request
 * larger than the whole budget runs alone.  So requests that arrive while others
 * are on the GPU join a running batch as soon as a slot and memory free up
 * (continuous batching), and a solve that finishes leaves it at once.  Solves of
 * at most 40^3 voxels run in a second batch on a stream of the highest priority,
 * with rounds of their own, so small requests are not paced by the largest ones.
 * The batch of larger solves holds at most 2 x 64^3 voxels at once (a larger
 * solve runs alone in it): one such solve already fills the GPU, so the queue's
 * shortest requests finish first instead of all of them sharing the device.
 * A solve's results do not depend on what else runs beside it. */
typedef struct evp_server evp_server;

typedef struct evp_status {
    int state;             /* 0 queued, 1 running, 2 done */
    int status;            /* when done: 0 or a status code as evp_solve_file returns */
    int macrosteps;        /* macrosteps completed */
    int n1, n2, n3;        /* grid */
    long long voxel_iters; /* voxels x equilibrium iterations executed */
    double queued_s;       /* submit -> admission */
    double run_s;          /* admission -> files written */
    double latency_s;      /* submit -> files written */
    unsigned long long footprint_bytes; /* device-memory estimate used for admission */
    char error[256];       /* message when status != 0 */
} evp_status;

/* hbm_budget_bytes: device memory the running solves may hold together (0: 85 % of
 * the free memory at open).  max_inflight: solves run at once (<= 0: 16).
 * tune_cache: the tile cache of the FFT passes (as evp_tune_cache); may be NULL. */
int evp_server_open(unsigned long long hbm_budget_bytes, int max_inflight, const char* tune_cache, evp_server** out);
/* Queue one solve (same deck and flags as evp_solve_file; precision 0 = plain FP64,
 * 1 = mixed precision as EVP_MIXED).
 * flags: EVP_WRITE_FILES (results, diagnostics and VTK, as the executable) or
 * EVP_WRITE_CSV (results and diagnostics only).  The ticket identifies it. */
int evp_submit(evp_server* srv, const char* fft_in, const char* out_dir, int mix, int modal, int precision, int flags,
               unsigned long long* ticket);
/* evp_submit with a wall-clock budget: deadline_s seconds from the solve's admission
 * (<= 0: none); a solve that overruns it ends between equilibrium iterations with
 * status -8 while the other solves continue. */
int evp_submit_deadline(evp_server* srv, const char* fft_in, const char* out_dir, int mix, int modal, int precision,
                        int flags, double deadline_s, unsigned long long* ticket);
/* Current state of a request (non-blocking). */
int evp_poll(evp_server* srv, unsigned long long ticket, evp_status* st);
/* Block until the request is done or timeout_s passes (timeout_s < 0: no limit);
 * returns 0 when done, 1 on timeout. */
int evp_wait(evp_server* srv, unsigned long long ticket, double timeout_s, evp_status* st);
/* Let queued and running solves finish, then release the server. */
int evp_server_close(evp_server* srv);

/* Message of the last failing call on this thread. */
const char* evp_last_error(void);
int evp_version(void);

#ifdef __cplusplus
}
#endif
#endif
