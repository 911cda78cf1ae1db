/* ug.h -- C ABI of the B200 RSA worldline packer (libug.so).
 *
 * Plain C types only; no torch or CUDA types in the signatures.  Every call
 * returns a status (UG_OK or a UG_E* code) and never exits the process; the
 * message of the last failure on the calling thread is in ug_last_error().
 *
 * Each entry point replaces one interface of the reference engines
 * (universe-analysis/universe-generator); the reference location is cited
 * beside it.  The reference engines are standalone programs driven through
 * argv, stderr and CSV files (braidlab/engine.py:50-112); this library is the
 * in-process form of the same contract, and ugb200.cli wraps it back into a
 * braid_cuda-compatible command line.
 */
#ifndef UG_H
#define UG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (the engines' fail-fast exits, cuda/braid_cuda.cu:597-636) */
#define UG_OK 0
#define UG_EINVAL 1     /* bad configuration (flag validation, braid_cuda.cu:597-636) */
#define UG_ENOMEM 2     /* device allocation failed */
#define UG_ECAP 3       /* a capacity was exceeded (never a silent drop) */
#define UG_ECUDA 4      /* CUDA runtime error */
#define UG_ETIMEDOUT 5  /* a bounded device wait gave up */
#define UG_ENOTSUP 6    /* combination not supported */

/* ---- model conventions */
#define UG_RNG_PHILOX 0 /* counter-based Philox4x32-10 candidate stream (this packer) */
#define UG_RNG_KNOT 1   /* xoshiro256** per attempt index, cuda/braid_knot.cu:207 */
#define UG_ZGRID_REF 0  /* z_t = (t+1) pi / (T+1), cuda/braid_cuda.cu:653-660 */
#define UG_ZGRID_MID 1  /* z_t = (t+1/2) pi / T */
#define UG_EXCL_REF 0   /* Chebyshev |d| <= 2/T per timestep, cuda/braid_cuda.cu:451,604 */
#define UG_EXCL_OPEN 1  /* Chebyshev |d| <  1/F per timestep */
#define UG_GROUP_NONE 0    /* unique packing */
#define UG_GROUP_SUBPATH 1 /* uniques, then subpaths joining one group (--subpaths,
                              cuda/braid_cuda.cu:46-58, 949-1043) */
#define UG_GROUP_UNIQUE 2  /* one phase: no contact founds a group, one group joins,
                              two or more reject */
#define UG_PREC_FP64 0  /* plain FP64 single-pass prefilter */
#define UG_PREC_MIXED 1 /* tensor-core split-BF16 prefilter + FP64 guard-band retest */

/* One universe (one reference engine run).  Mirrors the engine flags
 * -t, --terms, --seed, --attempts, --max-n, --until-accept-rate, --pin-sin1,
 * --subpaths, --sub-attempts, --sub-until-accept-rate
 * (cuda/braid_cuda.cu:534-584; cuda/braid_cuda3d.cu:862-913). */
typedef struct ug_universe_cfg {
    int32_t dim;        /* spatial axes, 1..3 (braid_cuda: 2, braid_cuda3d: 3) */
    int32_t T;          /* timesteps; the max frequency is T (braid_cuda.cu:597-603) */
    int32_t terms;      /* sinusoid terms per axis incl. sin1; 0 = full band (T) */
    int32_t rng;        /* UG_RNG_* */
    int32_t zgrid;      /* UG_ZGRID_* */
    int32_t excl;       /* UG_EXCL_* */
    int32_t cross1d;    /* 1+1D: also reject a sign change of the separation between steps */
    int32_t pin_sin1;   /* --pin-sin1 (braid_cuda.cu:170-188) */
    int32_t group_mode; /* UG_GROUP_* */
    int32_t round_size; /* candidates per round; 0 = 65536.  Results do not depend on it */
    uint64_t seed;
    int64_t attempts;     /* candidate budget of phase 1 */
    int64_t max_n;        /* --max-n: phase-1 unique cap (0 = off) */
    int64_t sub_attempts; /* --sub-attempts (0 = same as attempts) */
    double accept_rate;   /* --until-accept-rate (0 = off), braid_cuda.cu:931-943 */
    double sub_accept_rate;
    double sub_fill_rate; /* --sub-until-fill-rate: phase-2 stop on windowed newly occupied
                             grid cells per attempt (0 = off), braid_cuda.cu:960-1035 */
    int32_t euclid;       /* --euclid-collision: exclusion by the L2 ball of radius cell
                             instead of the Chebyshev cube (braid_cuda3d.cu:605-608) */
    int32_t surv_cap;     /* survivors resolved per round, at most 8192 (0 = 2^20 / T, 256 for
                             1+1D); a round is cut at the first survivor beyond it.  Results do
                             not depend on it */
} ug_universe_cfg;

typedef struct ug_run_opts {
    int32_t precision;       /* UG_PREC_* */
    int32_t device;          /* CUDA device ordinal (-1 = current) */
    int32_t rounds_per_sync; /* rounds per CUDA-graph replay / host status check (0 = 8) */
    int32_t use_graph;       /* capture the round sequence as a CUDA graph */
    int32_t kernel_timing;   /* record per-kernel CUDA events (no graph) */
    int32_t force_hash;      /* 1 = hashed collision grid even where a dense one fits */
    uint64_t stream;         /* cudaStream_t to run on (0 = library-owned stream) */
    int64_t slot_hint;       /* initial accepted-path capacity per universe (0 = auto) */
} ug_run_opts;

/* Per-universe result (the engine's stderr "done:" line and curve end point,
 * braid_cuda.cu:945, 1039-1042). */
typedef struct ug_stats {
    int64_t n;          /* accepted paths (uniques + subpaths) */
    int64_t n_unique;   /* uniques / groups founded */
    int64_t n_sub;      /* subpaths */
    int64_t attempts;   /* candidates decided (all phases) */
    int64_t phase1_end; /* first candidate index of the subpath phase */
    int64_t rounds;
    int64_t gray;       /* mixed precision: candidates re-tested in FP64 */
    int64_t evals;      /* prefilter position evaluations (candidate x timestep) */
    int64_t evals_fp64; /* of which in FP64 */
    int32_t state;      /* 1 = done */
    int32_t grid_kind;  /* 0 dense, 1 hash */
    int64_t filled;     /* occupied (timestep, cell) buckets of the collision grid
                           (the `filled` of braid_cuda.cu:695, 877) */
    int64_t visits;     /* accepted points examined by the prefilter's neighbour tests */
} ug_stats;

/* Per-kernel device time accumulated while kernel_timing is on. */
typedef struct ug_kernel_times {
    double ms[12];
    int64_t launches[12];
    const char* names[12];
} ug_kernel_times;

/* Library version (ABI revision). */
int ug_version(void);

/* Message of the last failure on this thread; returns its length. */
int ug_last_error(char* buf, size_t len);

/* sizeof of the structs a binding must lay out, in this order: ug_universe_cfg,
 * ug_run_opts, ug_stats, ug_kernel_times, ug_hit, ug_frames_cfg, ug_frames_out.
 * Writes min(n, 7) of them and returns 7.  Lets a binding (ctypes, cffi, cgo)
 * check its struct definitions against the library it loaded; no device work.
 * No reference counterpart (the engines' interface is argv and files). */
int ug_struct_sizes(int64_t* sizes, int32_t n);

/* Name ("<device name> sm_XY") and SM count of a CUDA device (-1: the current
 * one); the autotuner keys its cache by them.  No reference counterpart. */
int ug_device_info(int32_t device, char* name, size_t len, int32_t* sms);

/* Self-test of the bounded device waits (no reference counterpart): a kernel
 * waits on an mbarrier that nothing completes, with the wait routine of the
 * tensor-core prefilter and a limit of limit_ns (at most 10 s); the wait gives
 * up and the kernel stores UG_ETIMEDOUT in *status and returns, leaving the
 * context usable.  Returns UG_OK when the kernel ran. */
int ug_selftest_bounded_wait(int64_t limit_ns, int32_t* status);

/* Create a batch of independent universes on one GPU (replaces one engine
 * process per job, braidlab/orchestrator.py:85-147).  The library owns all
 * device memory inside the handle. */
int ug_batch_create(const ug_universe_cfg* cfgs, int32_t n, const ug_run_opts* opts, void** out);

/* Run every universe to its stop rule (the round loops of
 * cuda/braid_cuda.cu:885-944 and :949-1043, cuda/braid_knot.cu:401-469).
 * max_rounds > 0 bounds the number of rounds; returns UG_OK while work
 * remains (check ug_batch_done). */
int ug_batch_run(void* h, int64_t max_rounds);

/* Restart every universe from an empty packing, keeping all allocations;
 * seeds (n values, may be NULL) replace the candidate-stream seeds.  A fresh
 * engine run per job (braidlab/orchestrator.py:85-147) without re-allocation. */
int ug_batch_reset(void* h, const uint64_t* seeds);

/* 1 when every universe has stopped, 0 otherwise (negative on error). */
int ug_batch_done(void* h);

/* Result counters of universe u (braid_cuda.cu:945 "done: N=.. in .. attempts"). */
int ug_batch_stats(void* h, int32_t u, ug_stats* out);

/* Accepted candidate indices (admission order) and group ids of universe u.
 * Size query: pass cap = 0 and read *n. */
int ug_batch_accepted(void* h, int32_t u, int64_t* idx, int32_t* gid, int64_t cap, int64_t* n);

/* Accepted candidate indices and group ids of every universe in one call:
 * counts[u] (n entries) gets each universe's count, idx / gid (cap entries,
 * either may be NULL) the lists concatenated in universe order.  A device-side
 * gather, then one copy per array (the admission logs of all jobs of a
 * campaign, cuda/braid_knot.cu:449-460, read back at once).  Size query:
 * cap = 0. */
int ug_batch_accepted_all(void* h, int64_t* idx, int32_t* gid, int64_t cap, int64_t* counts);

/* Wrapped comoving positions [n][dim][T] of the accepted paths (FP64),
 * the trajectories evalPath fills (braid_cuda.cu:831-862). */
int ug_batch_positions(void* h, int32_t u, double* pos, int64_t cap_paths);

/* Worldline parameters of the accepted paths, the --dump-params content
 * (braid_cuda.cu:1062-1104; braid_cuda3d.cu:1578-1613): per path and axis
 * a2, then nw terms of (a, b, f) in term order. a2 [n][dim], a/f [n][dim][nw],
 * b [n][dim][nw]. */
int ug_batch_params(void* h, int32_t u, double* a2, double* a, int32_t* b, double* f,
                    int64_t cap_paths);

/* The same worldline parameters as ug_batch_params, produced without
 * allocating any device memory: the regenerated parameters are staged in a
 * fixed 16 MiB buffer that the library image reserves on every GPU that
 * loads it, then copied to the caller's host buffers.  No counterpart in
 * the reference.  For callers that cannot call cudaMalloc at the time of the
 * call -- a serving process that reserved all of its device memory at
 * start-up, or a host whose allocator policy forbids allocations after
 * start-up.  Dumps needing more than 16 MiB (paths x dim x (8 + 20 nw)
 * bytes) fail with UG_ECAP.  The first call on a device looks up the
 * buffer's device address; make it before any stream capture.  All calls
 * share the buffer: calls whose work overlaps on the GPU race. */
int ug_batch_params_noalloc(void* h, int32_t u, double* a2, double* a, int32_t* b, double* f,
                            int64_t cap_paths);

/* Per-kernel device times (kernel_timing = 1). */
int ug_batch_kernel_times(void* h, ug_kernel_times* out);

/* Kernels launched by the batch so far and bytes it copied host->device and
 * device->host (cumulative). */
int ug_batch_counters(void* h, int64_t* launches, int64_t* h2d_bytes, int64_t* d2h_bytes);

/* Reset the per-kernel timers. */
int ug_batch_reset_times(void* h);

/* Maximum |X_mixed - X_fp64| of the tensor-core evaluation over the first
 * `count` candidates of universe u (all timesteps and axes): the achieved
 * position error of the mixed-precision prefilter against FP64.  Also
 * returns the widest guard band the prefilter applies (`margin`) and the
 * largest ratio of the error to the guard band of its own (candidate,
 * timestep) (`max_ratio`, below 1 whenever every decision is exact). */
int ug_batch_mixed_error(void* h, int32_t u, int64_t first, int64_t count, double* max_err,
                         double* margin, double* max_ratio);

/* ---- checkpoint / resume of a run (in-run counterpart of the store's job-level
 * resume, braidlab/store.py:89-108).  A checkpoint of universe u is its
 * admissions (ug_batch_accepted: candidate indices in admission order and their
 * groups) plus an opaque state block of ug_state_bytes() bytes
 * (ug_batch_save_state): round position, counters, stop windows.  Because the
 * candidate stream is counter-based, ug_batch_restore rebuilds the packing from
 * the admissions alone (trajectories regenerated, grid re-appended in admission
 * order) and the run continues exactly as if it had not stopped, in this or any
 * other batch holding a universe of the same model and seed. */
int64_t ug_state_bytes(void);
int ug_batch_save_state(void* h, int32_t u, void* state);
int ug_batch_restore(void* h, int32_t u, int64_t n, const int64_t* idx, const int32_t* gid, const void* state);

/* --diag probe (braid_cuda3d.cu:1645-1667): n fresh candidates of the stream keyed
 * by `seed` (the run's own stream uses the universe seed) tested against the
 * current packing without admitting any; proposed / accepted counts per bin of
 * the x axis's sin1 offset a2 over [-1, 1), `bins` bins. */
int ug_batch_probe(void* h, int32_t u, uint64_t seed, int64_t n, int32_t bins, int64_t* proposed,
                   int64_t* accepted);

/* Release all device memory of the batch. */
int ug_batch_destroy(void* h);

/* ---- frames: past-light-cone images of a packing (cuda/frame_bake.cu) */

/* One image of a worldline on the front (the BRF1 hit record, frame_bake.cu:31-40). */
typedef struct ug_hit {
    uint32_t src;  /* source path (dump row) */
    float dx, dy;  /* offset from the pulse centre (torus image included) */
    float chi;     /* front radius at emission */
    float z_emit;  /* conformal time of emission */
} ug_hit;

/* frame_bake's flags (frame_bake.cu:431-470). */
typedef struct ug_frames_cfg {
    int32_t front;         /* 0 speed, 1 fit, 2 budget */
    int32_t cheb;          /* 1 square (Chebyshev) metric, 0 circle; budget forces 1 */
    int32_t n_frames;      /* instants z_obs spread over [from, to] */
    int32_t wraps;         /* torus image cap K; -1 = ceil((chi_max + 4) / 2) */
    double from_pi, to_pi; /* z_obs range, units of pi */
    double zmin_pi;        /* rewind floor, units of pi */
    double speed;          /* conformal front speed (front 0) */
    int32_t n_obs;
    int32_t density_bins;  /* > 0: histogram hit offsets into bins x bins per (frame, observer) */
    const int32_t* obs_type; /* [n_obs] 0 path observer, 1 comoving point */
    const int32_t* obs_path; /* [n_obs] path index (type 0) */
    const double* obs_xy;    /* [n_obs][2] point (type 1) */
} ug_frames_cfg;

typedef struct ug_frames_out {
    ug_hit* hits;        /* all hits, (frame, observer)-major, each group sorted by (chi, src) */
    int64_t hit_cap;
    int64_t* hit_count;  /* [n_frames][n_obs] */
    double* frame_meta;  /* [n_frames][3]: z_obs, chi_max, K */
    double* obs_meta;    /* [n_frames][n_obs][4]: ox, oy, beta_x, beta_y */
    uint32_t* density;   /* [n_frames][n_obs][bins][bins] over [-chi_max, chi_max]^2, or NULL */
    int64_t hits_total;  /* out: hits found (also when hit_cap is too small) */
} ug_frames_out;

/* Bake frames of a 2+1 packing given as dump arrays: a2 [n][2], a/b/f
 * [n][2][nw] (the frame_bake driver, frame_bake.cu:398-635: load_dump,
 * grid_kernel, hits_kernel, BRF1 writer; plus the density scatter). */
int ug_frame_bake(const ug_frames_cfg* cfg, int32_t n, int32_t nw, const double* a2, const double* a,
                  const double* b, const double* f, ug_frames_out* out);

/* Bake frames of the accepted paths of universe u of a batch (2+1) straight from
 * the device: the packer's parameters never leave the GPU (the reference's
 * dump CSV -> frame_bake pipeline, frame_bake.cu:398-635, without the file).
 * Path p of the frames is the p-th admission (the dump row order).  With
 * out->hits == NULL only hit counts and densities come back. */
int ug_batch_frames(void* h, int32_t u, const ug_frames_cfg* cfg, ug_frames_out* out);

/* Observer-view remap of one frame's hits, the viewer's draw-time transform
 * (braidlab/frames.py:147-188, apparent_positions).  UG_VIEW_STATIC: the stored
 * offsets and ln_dopp = 0.  UG_VIEW_MOVING: beta is capped at |beta| = 0.995 (and
 * |beta| <= 1e-6 is static); each hit's unit direction n is boosted into the
 * observer's rest frame, n' = [n + gamma beta + (gamma - 1)(u.n) u] / [gamma (1 +
 * beta.n)] with u = beta / |beta|, ln_dopp = ln(gamma (1 + beta.n)), and the image is
 * put back at its own chi on the Chebyshev shell (cheb != 0) or the Euclidean one;
 * hits at the pulse centre keep their offsets.  Outputs are n doubles each.  Host
 * buffers, computed on the GPU; UG_EINVAL for another mode. */
#define UG_VIEW_STATIC 0
#define UG_VIEW_MOVING 1
int ug_apparent_positions(const ug_hit* hits, int64_t n, double beta_x, double beta_y, int32_t mode,
                          int32_t cheb, double* ax, double* ay, double* ln_dopp);
/* The same on device buffers (hits as from a frame bake left on the GPU), enqueued
 * on `stream` (a cudaStream_t; NULL: the legacy default stream). */
int ug_apparent_positions_async(const ug_hit* d_hits, int64_t n, double beta_x, double beta_y,
                                int32_t mode, int32_t cheb, double* d_ax, double* d_ay,
                                double* d_ln_dopp, void* stream);

/* ---- single-universe convenience: a batch of one (the ug_pack_* surface) */
int ug_pack_create(const ug_universe_cfg* cfg, const ug_run_opts* opts, void** out);
int ug_pack_run(void* h);
int ug_pack_stats(void* h, ug_stats* out);
int ug_pack_destroy(void* h);

#ifdef __cplusplus
}
#endif
#endif
