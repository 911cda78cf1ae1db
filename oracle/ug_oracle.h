/* ug_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the reference's RSA worldline-packing path, used as the
 * parity checker for the CUDA packer.  Only tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline / --impl reference legs may load it; the
 * product never links or calls it.
 *
 * Parity pins: the knot-mode candidate stream and admission are checked
 * against outputs of the reference's own code (cuda/braid_knot.cu compiled
 * from the reference tree, see oracle/ref/ and tests/golden/).  The Philox
 * mode has no reference counterpart; it is pinned through the published
 * Philox4x32-10 known-answer vectors and cross-checked against the knot mode
 * through shared evaluation / admission code.
 */
#ifndef UG_ORACLE_H
#define UG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORA_RNG_PHILOX 0
#define ORA_RNG_KNOT 1
#define ORA_ZGRID_REF 0 /* z_t = (t+1) pi / (T+1)  (braid_knot.cu:311) */
#define ORA_ZGRID_MID 1 /* z_t = (t+0.5) pi / T                      */
#define ORA_EXCL_REF 0  /* Chebyshev |d| <= 2/T    (braid_knot.cu:239) */
#define ORA_EXCL_OPEN 1 /* Chebyshev |d| <  1/F                      */

#define ORA_GROUP_NONE 0    /* plain unique packing                         */
#define ORA_GROUP_SUBPATH 1 /* reference two-phase: uniques, then subpaths  */
#define ORA_GROUP_UNIQUE 2  /* one phase: 0 contacts -> new group, 1 -> join */

#define ORA_MAX_F 512

typedef struct ora_model {
    int32_t dim;     /* spatial axes, 1..3 */
    int32_t T;       /* timesteps; max frequency F = T */
    int32_t nw;      /* wiggle terms per axis (F-1 = full band) */
    int32_t rng;     /* ORA_RNG_* */
    int32_t zgrid;   /* ORA_ZGRID_* */
    int32_t excl;    /* ORA_EXCL_* */
    int32_t cross1d; /* 1+1D sign-change (crossing) rejection */
    int32_t pin;     /* --pin-sin1: sin1 amplitudes forced to zero */
    int32_t euclid;  /* --euclid-collision: L2 ball instead of the Chebyshev cube */
    uint64_t seed;
} ora_model;

typedef struct ora_run {
    int64_t attempts;     /* candidate budget of the (first) phase */
    int64_t max_n;        /* stop phase 1 at this many paths (0 = off) */
    int32_t group_mode;   /* ORA_GROUP_* */
    int32_t nthreads;     /* 0/1 = sequential RSA; >1 = threaded batch prefilter + in-order decisions */
    int64_t sub_attempts; /* subpath-phase budget (ORA_GROUP_SUBPATH) */
    int64_t round;        /* batch size of the threaded form */
    double accept_rate;     /* phase-1 windowed accept-rate stop (0 = off) */
    double sub_accept_rate; /* phase-2 windowed accept-rate stop (0 = off) */
    double sub_fill_rate;   /* phase-2 windowed new-volume stop (0 = off) */
} ora_run;

typedef struct ora_result {
    int64_t cap;          /* capacity of acc_idx / gid (in) */
    int64_t* acc_idx;     /* accepted candidate indices, admission order (out) */
    int32_t* gid;         /* group label per accepted path (out, may be NULL) */
    int64_t n_acc;        /* accepted paths (out) */
    int64_t n_unique;     /* uniques / groups founded (out) */
    int64_t n_sub;        /* subpaths (out) */
    int64_t attempts;     /* candidates consumed, all phases (out) */
    int64_t phase1_end;   /* first candidate index of the subpath phase (out) */
} ora_result;

/* Philox4x32-10 block function (Salmon, Moraes, Dror, Shaw, SC'11). */
void ora_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* xoshiro256** seeded by splitmix64: the first n outputs for `seed`. */
void ora_xoshiro_stream(uint64_t seed, int32_t n, uint64_t* out);

/* One candidate.  b/a/f are [dim][nw] in draw order, a2 is [dim];
 * alpha/beta are the canonical frequency-indexed coefficients [dim][T+1]
 * (alpha_b = sum a cos f, beta_b = sum a sin f over terms of frequency b). */
int ora_candidate(const ora_model* m, uint64_t idx, int32_t* b, double* a, double* f, double* a2,
                  double* alpha, double* beta);

/* Wrapped comoving positions [dim][T] of candidate idx (FP64). */
int ora_positions(const ora_model* m, uint64_t idx, double* pos);

/* z grid, sin(b z), cos(b z) tables as the packer uploads them:
 * z[T], invsinz[T], S[(T+1)*T], C[(T+1)*T] (row b, column t). */
int ora_tables(const ora_model* m, double* z, double* invsinz, double* S, double* C);

/* Full packing run. */
int ora_pack(const ora_model* m, const ora_run* run, ora_result* res);

/* Positions of the accepted paths of the last ora_pack call on this thread
 * are not kept; callers recompute them with ora_positions. */

#ifdef __cplusplus
}
#endif
#endif
