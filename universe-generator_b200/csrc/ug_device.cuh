// ug_device.cuh -- device-side model of the RSA worldline packer.
//
// A worldline axis is x(z) = sum_b a_b [sin(b z + f_b) - sin f_b] + a2 sin z
// (cuda/braid_cuda.cu:8-16).  The packer evaluates the comoving position
// X(z_t) = x(z_t) / sin z_t in the sine basis
//     X_t = wrap( a2 + invsinz_t * sum_{b=2..F} (alpha_b S_bt + beta_b Cm_bt) )
// with alpha_b = a_b cos f_b, beta_b = a_b sin f_b (zero for odd b),
// S_bt = sin(b z_t) and Cm_bt = cos(b z_t) - 1 (host-built FP64 tables, the
// table form of cuda/braid_knot.cu:211-230).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace ug {

// Index guard.  The product build compiles UG_IDX(i, n) to i.  The checked
// build (-DUG_CHECKED) records the first out-of-range index (source line,
// index, bound) in ug_check_record and substitutes 0, so a bad index is
// reported instead of dereferenced.
#ifdef UG_CHECKED
extern __device__ unsigned long long ug_check_record[4];
__device__ __noinline__ static int64_t ug_idx_fail(int64_t i, int64_t n, int line) {
    if (atomicCAS(&ug_check_record[0], 0ull, (unsigned long long)line) == 0ull) {
        ug_check_record[1] = (unsigned long long)i;
        ug_check_record[2] = (unsigned long long)n;
        ug_check_record[3] = 1ull;
    }
    return 0;
}
__device__ __forceinline__ int64_t ug_idx(int64_t i, int64_t n, int line) {
    return ((uint64_t)i < (uint64_t)n) ? i : ug_idx_fail(i, n, line);
}
#define UG_IDX(i, n) ::ug::ug_idx((int64_t)(i), (int64_t)(n), __LINE__)
#else
#define UG_IDX(i, n) (i)
#endif

constexpr double kPi = 3.14159265358979323846;
constexpr int kMaxF = 256;        // max frequency / timesteps per universe
constexpr int kTile = 128;        // candidates per prefilter tile
enum : int { kConflictCap = 48 };  // earlier in-round conflicts kept per survivor
enum : int { kSmaxCap = 8192 };    // survivors resolved per universe per round (max)
constexpr uint32_t kEmptyKey32 = 0xffffffffu;
constexpr uint64_t kEmptyKey = ~0ull;

enum RngMode : int32_t { RNG_PHILOX = 0, RNG_KNOT = 1 };
enum GroupMode : int32_t { GROUP_NONE = 0, GROUP_SUBPATH = 1, GROUP_UNIQUE = 2 };
enum GridKind : int32_t { GRID_DENSE = 0, GRID_HASH = 1 };

// Universe state flags (UniCtl::state)
enum : int32_t { ST_ACTIVE = 0, ST_DONE = 1, ST_GROW = 2, ST_ERROR = 3 };

// One accepted (or in-round survivor) point: FP64 position, chain link, group.
struct __align__(32) Pt64 {
    double c[3];
    int32_t next;
    int32_t gid;
};
// FP32 copy used by the mixed-precision prefilter.
struct __align__(16) Pt32 {
    float c[3];
    int32_t next;
};

// Read-only per-universe description (device copy lives in UniDev array).
struct UniDev {
    // model
    int32_t dim, T, F, nw;
    int32_t rng, inclusive, cross1d, pin;
    int32_t group_mode;  // GroupMode; GROUP_SUBPATH runs phase 1 as NONE then 2 as SUBPATH
    int32_t gw;          // cells per axis
    uint64_t seed;
    double cell;         // exclusion radius == cell width
    uint32_t modmax;     // knot: frequencies drawn in [2, modmax+1]
    int32_t B_max;       // candidates per round cap
    int32_t S_max;       // survivors per round cap
    int32_t euclid;      // exclusion by the L2 ball of radius cell (else the Chebyshev cube)
    // tables
    const double* S;       // [(F+1) * T]
    const double* Cm;      // [(F+1) * T]
    const double* invsinz; // [T]
    const int32_t* order;  // [T] endpoint-first
    // main grid
    int32_t grid_kind;
    int32_t rblock_shift;  // round table: blocks of 2^rblock_shift cells per axis
    int32_t* heads;        // dense: chain heads [T * gw^dim]
    ulonglong2* hslot;     // hash [hcap]: x = key t<<40 | cell, y = head slot (low 32 bits)
    uint64_t hmask;        // hcap - 1
    // occupancy bitmap: one bit per (timestep, coarse cell); a coarse cell is
    // 2^occ_shift cells per axis.  A clear bit proves the cells empty, so
    // empty neighbourhoods cost one L2-resident word instead of a grid probe.
    // 3+1 lays the bits out in 4x4x4 bricks and 2+1 in 8x8 bricks, one 64-bit
    // word per brick, so a 3x3x3 neighbourhood reads ~3.4 words instead of ~9 rows
    uint32_t* occ;
    int32_t occ_shift;
    int32_t occ_gw;        // coarse cells per axis
    int64_t occ_per_t;     // coarse cells (2+1, 3+1: bricks) per timestep
    // dilated first-level filter: one bit per (timestep, block of 2^occ1_shift
    // fine cells per axis), set for every block holding a cell that meets the
    // cube of half-width occ1_reach (the exclusion radius plus the widest guard
    // band, plus rounding slack) around a committed point.  A test point within
    // radius + band of some point therefore has its own cell's block marked: a
    // clear bit proves that no point is near enough to count, with ONE load.
    uint32_t* occ1;
    int32_t occ1_gw;       // blocks per axis
    int32_t occ_nb;        // 2+1 and 3+1: bricks per axis
    int64_t occ1_per_t;
    int32_t occ1_shift;
    // main hash keyed by coarse cells of 2^gkey_shift cells per axis (those of the
    // occupancy bitmap; 0 = cells).  A coarse key's slot carries the complement of
    // its cells' occupancy mask in the high half of y.
    int32_t gkey_shift;
    double occ1_reach;
    // accepted points
    Pt64* pts;             // [slot_cap * T]
    Pt32* ptf;             // [slot_cap * T]
    int64_t slot_cap;
    // per-round buffers
    uint32_t* surv_bits;   // [B_max / 32]
    uint32_t* gray_bits;   // [B_max / 32]
    int32_t* g0;           // [B_max]  group mode: single pre-round group touched (-1 none)
    int32_t* surv_off;     // [S_max]  candidate offset within the round
    int32_t* gray_off;     // [B_max]  mixed: offsets of candidates sent to the FP64 retest
    Pt64* spos;            // [S_max * T]
    uint64_t* rhead;       // round table [T * rblocks]: epoch<<32 | head survivor rank of
                           // each (timestep, block); entries of other epochs are empty
    int64_t rblocks;       // blocks per timestep (rblock_gw^dim)
    int32_t* ccount;       // [S_max]
    int32_t* clist;        // [S_max * kConflictCap]
    int32_t* sgid;         // [S_max]  resolved group / -1 rejected, -2 unresolved
    int32_t* acc_rank;     // [S_max]  slot offset of accepted survivors, -1 otherwise
    int64_t* acc_idx;      // [slot_cap] candidate index of each accepted slot
    // mixed-precision (tensor-core) prefilter
    const uint8_t* mx_bimg;  // split-BF16 sine-basis table, one UMMA image per K chunk
    int32_t mx_ok;           // universe runs the tensor-core prefilter
    int32_t mx_chunks;       // K chunks of 48 coefficient entries (16 frequency pairs)
    int32_t mx_tpad;         // timesteps padded to 16 (B rows)
    int32_t mx_nmma;         // UMMA N per pass
    int32_t mx_npass;        // timestep passes (2 when dim * tpad > 512 TMEM columns)
    float mx_margin;         // guard band of the FP32 Chebyshev test
    // per-(candidate, timestep) guard band: 2 mx_mc1 * bound + mx_mc0, where
    // bound = min(2, 2 invsinz_t rho) >= sum_k |A_k B_kt| / sum E and
    // rho = sum_b (E_b / b) / sum E of the candidate (largest over its axes)
    float mx_mc1, mx_mc0;
    // survivor trajectories as an FP64 product coef[K x Rpad]^T * KT[K x Tpad]:
    // term k runs over (b = 2..F: sin term, then the cos term of even b) -- the
    // accumulation order of eval64, so both give the same bits
    const double* KT;        // [K * Tpad] S_b / Cm_b rows in term order, zero padded
    double* coef;            // [K * Rpad] alpha_b / beta_b of row (survivor r, axis) = r * dim + ax
    double* a2row;           // [Rpad]
    int32_t K, Tpad, Rpad, pad4;
    // sizes (index guards of the checked build)
    int64_t occ_words, occ1_words, dense_cells, bimg_bytes;
};

// Mutable per-universe control block (device).
struct UniCtl {
    int64_t next_cand;     // first candidate of the next round
    int64_t phase_end;     // candidate index where the current phase ends
    int64_t sub_budget;    // GROUP_SUBPATH: candidates of phase 2
    int64_t max_n;         // phase-1 unique cap (0 = off)
    int64_t round_base;    // this round: candidates [round_base, round_base + B)
    int64_t n_slots;       // accepted paths (== slots used)
    int64_t n_unique, n_sub;
    int64_t attempts;      // candidates fully decided
    int64_t phase1_end;
    int32_t B;             // this round's candidate count
    int32_t round_B;       // adaptive round size
    int32_t S;             // survivors this round (after truncation)
    int32_t S_raw;         // survivors found by the prefilter
    int32_t trunc;         // survivor rank where the round was truncated (S if none)
    int32_t phase;         // 1 or 2
    int32_t state;         // ST_*
    int32_t epoch;         // round-table epoch
    int32_t n_gray;        // mixed: candidates sent to the FP64 retest this round
    int32_t accepted_round;
    int64_t gray_total;    // mixed: FP64 retests over the run
    int64_t rounds;
    int64_t hash_used;     // main grid hash entries in use
    int64_t n_slots_prev;  // n_slots before this round's commit
    int64_t evals;         // prefilter (candidate, timestep) position evaluations
    int64_t visits;        // prefilter: accepted points examined by the neighbour tests
    int64_t evals_fp64;    // of which evaluated in FP64 (plain path / guard-band retest)
    int32_t stop_at;       // survivors [0, stop_at) resolved this round
    int32_t tile_ns;       // mixed prefilter: slowest tile of the last round (ns), orders the next round's tiles
    int32_t B_min, B_cap;  // round-size adaptation bounds
    int32_t err_code;
    int32_t pad;
    // windowed stops (braid_cuda.cu:585-590, 931-943 and the phase-2 new-volume
    // window of :953-1037).  Each window is 32 buckets of q = win_target / 32
    // candidates aligned at the phase start (phase_start); rounds never straddle a
    // bucket boundary, and at each boundary the phase ends when 32 buckets exist,
    // more than 1e6 candidates are decided and the last 32 buckets' count over
    // 32 q is below the threshold.  win_*: admissions (accept rate, phase 1 or 2),
    // fwin_*: newly occupied grid cells (phase 2).
    double accept_rate;     // phase 1 threshold (0 = off)
    double sub_accept_rate; // phase 2 threshold (0 = off)
    double win_thr;         // threshold of the running phase
    int64_t phase_start;    // first candidate of the running phase
    int64_t win_q, win_nb, win_sum, win_cur;
    int64_t win_ring[32];
    // occupied (timestep, cell) buckets of the collision grid
    int64_t filled;         // occupied cells so far
    int64_t round_new;      // cells first occupied by this round's commit
    int64_t last_used;      // candidates decided by the last round
    double sub_fill_rate;   // threshold (0 = off)
    int64_t fwin_q, fwin_nb, fwin_sum, fwin_cur;
    int64_t fwin_ring[32];
};

// Bucket size of a window for threshold thr: win_target = clamp(30 / thr, 2e7, 5e9)
// candidates (braid_cuda.cu:589-590) in 32 buckets; 0 = off.
__host__ __device__ __forceinline__ int64_t win_bucket(double thr) {
    if (!(thr > 0)) return 0;
    double t = 30.0 / thr;
    t = t < 2e7 ? 2e7 : (t > 5e9 ? 5e9 : t);
    const int64_t W = (int64_t)t;
    return W / 32 > 0 ? W / 32 : 1;
}

// ------------------------------------------------------------------ helpers

__host__ __device__ __forceinline__ double torus_wrap(double x) {
    return x - 2.0 * floor((x + 1.0) * 0.5);
}
__host__ __device__ __forceinline__ double torus_delta(double d) {
    if (d > 1.0) return d - 2.0;
    if (d < -1.0) return d + 2.0;
    return d;
}
__device__ __forceinline__ float torus_wrapf(float x) {
    return x - 2.0f * floorf((x + 1.0f) * 0.5f);
}
__device__ __forceinline__ float torus_deltaf(float d) {
    if (d > 1.0f) return d - 2.0f;
    if (d < -1.0f) return d + 2.0f;
    return d;
}
__device__ __forceinline__ int cell_of(double X, double cell, int gw) {
    int c = (int)floor((X + 1.0) / cell);
    return c >= gw ? gw - 1 : (c < 0 ? 0 : c);
}
__device__ __forceinline__ bool hit1(double d, double cell, int inclusive) {
    const double ad = fabs(d);
    return inclusive ? ad <= cell : ad < cell;
}

// Exclusion test of two points: the Chebyshev cube of half-width cell, or the
// L2 ball dX*dX + dY*dY + dW*dW <= cell*cell (cuda/braid_cuda3d.cu:605-608),
// summed in that order without contraction so every decision matches the
// reference expression bit for bit.
__device__ __forceinline__ bool pair_hit64(const UniDev& U, const double* P, const double* Q) {
    if (!U.euclid) {
#pragma unroll
        for (int ax = 0; ax < 3; ax++)
            if (ax < U.dim && !hit1(torus_delta(P[ax] - Q[ax]), U.cell, U.inclusive)) return false;
        return true;
    }
    double s = 0.0;
#pragma unroll
    for (int ax = 0; ax < 3; ax++) {
        if (ax < U.dim) {
            const double d = torus_delta(P[ax] - Q[ax]);
            s = __dadd_rn(s, __dmul_rn(d, d));
        }
    }
    const double r2 = __dmul_rn(U.cell, U.cell);
    return U.inclusive ? s <= r2 : s < r2;
}

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw: "Parallel random numbers: as
// easy as 1, 2, 3", SC'11): 10 rounds of the 4x32 S-box with Weyl key bumps.
__host__ __device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
    for (int r = 0; r < 10; r++) {
        if (r) {
            k.x += 0x9E3779B9u;
            k.y += 0xBB67AE85u;
        }
#ifdef __CUDA_ARCH__
        const uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
#else
        const uint64_t p0 = (uint64_t)0xD2511F53u * c.x, p1 = (uint64_t)0xCD9E8D57u * c.z;
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
#endif
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    }
    return c;
}

// Counter layout of the Philox candidate stream: block p of axis ax of
// candidate idx.  Block 0 carries a2; block p >= 1 the frequency pair (2p, 2p+1).
__host__ __device__ __forceinline__ uint4 philox_block(uint64_t seed, uint64_t idx, int ax, int p) {
    return philox4x32_10(make_uint4((uint32_t)idx, (uint32_t)(idx >> 32),
                                    ((uint32_t)ax << 16) | (uint32_t)p, 0u),
                         make_uint2((uint32_t)seed, (uint32_t)(seed >> 32)));
}

// xoshiro256** + splitmix64 seeding: the reference's per-candidate stream
// (cuda/braid_knot.cu:56-90, seeded per attempt index as braid_knot.cu:207).
struct Xo {
    uint64_t s[4];
    __device__ __forceinline__ void seed(uint64_t sd) {
#pragma unroll
        for (int i = 0; i < 4; i++) {
            sd += 0x9E3779B97F4A7C15ULL;
            uint64_t z = sd;
            z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
            z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
            s[i] = z ^ (z >> 31);
        }
    }
    __device__ __forceinline__ uint64_t next() {
        const uint64_t x = s[1] * 5;
        const uint64_t result = ((x << 7) | (x >> 57)) * 9;
        const uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = (s[3] << 45) | (s[3] >> 19);
        return result;
    }
    __device__ __forceinline__ double f64() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
    __device__ __forceinline__ uint32_t below(uint32_t n) { return (uint32_t)(next() % n); }
    __device__ __forceinline__ bool flip() { return next() & 1ULL; }
};
__device__ __forceinline__ uint64_t knot_seed(uint64_t seed, uint64_t idx) {
    return seed ^ (idx * 0x9E3779B97F4A7C15ULL + 0x1234567ULL);
}

// ------------------------------------------------- FP64 candidate generation
// Writes the canonical coefficients of one axis into alpha/beta [F+1]
// (indices 2..F used) and returns a2.  `stride` lets the arrays live in
// shared memory interleaved across threads.

// Philox stream: E_b = -log((r + 1/2) 2^-32), w_b = E_b / sum_b E_b (ascending
// b), a_b = +-w_b / b, f_b = (r >> 1) 2^-31 pi on even b, a2 = r 2^-31 - 1.
__device__ __forceinline__ double gen_philox64(const UniDev& U, uint64_t idx, int ax, double* alpha,
                                               double* beta, int stride) {
    const int F = U.F;
    double a2 = 0.0;
    double sum = 0.0;
    for (int p = 0; 2 * p <= F; p++) {
        const uint4 o = philox_block(U.seed, idx, ax, p);
        if (p == 0) {
            a2 = U.pin ? 0.0 : (double)o.x * (1.0 / 2147483648.0) - 1.0;
            continue;
        }
        const int be = 2 * p, bo = 2 * p + 1;
        const double Ee = -log(((double)o.x + 0.5) * (1.0 / 4294967296.0));
        sum += Ee;
        alpha[be * stride] = (o.z & 1u) ? -Ee : Ee;  // sign folded in, phase parked in beta
        beta[be * stride] = (double)(o.z >> 1) * (1.0 / 2147483648.0) * kPi;
        if (bo <= F) {
            const double Eo = -log(((double)o.y + 0.5) * (1.0 / 4294967296.0));
            sum += Eo;
            alpha[bo * stride] = (o.w & 1u) ? -Eo : Eo;
        }
    }
    for (int b = 2; b <= F; b++) {
        const double e = alpha[b * stride];
        double amp = fabs(e) / sum / (double)b;
        if (e < 0.0 || (e == 0.0 && signbit(e))) amp = -amp;
        if (b & 1) {
            alpha[b * stride] = amp;
            beta[b * stride] = 0.0;
        } else {
            double sf, cf;
            sincos(beta[b * stride], &sf, &cf);
            alpha[b * stride] = amp * cf;
            beta[b * stride] = amp * sf;
        }
    }
    return a2;
}

// Knot stream (reference draw order, cuda/braid_knot.cu:111-166) for ALL axes.
// bj/aj/fj: scratch [nw] per axis (stride applies), coefficients accumulated
// into alpha/beta [dim][F+1] (row pitch F+1, stride applies).
__device__ inline void gen_knot64(const UniDev& U, uint64_t idx, double* alpha, double* beta,
                                  double* a2, int32_t* bj, double* wj, int stride) {
    Xo r;
    r.seed(knot_seed(U.seed, idx));
    const int nw = U.nw, F = U.F;
    for (int ax = 0; ax < U.dim; ax++) {
        double* al = alpha + (size_t)ax * (F + 1) * stride;
        double* bt = beta + (size_t)ax * (F + 1) * stride;
        for (int b = 0; b <= F; b++) al[b * stride] = bt[b * stride] = 0.0;
        if ((uint32_t)nw == U.modmax) {
            for (int j = 0; j < nw; j++) bj[j * stride] = j + 2;
            for (int j = nw - 1; j > 0; j--) {
                const int k = (int)r.below((uint32_t)(j + 1));
                const int32_t tmp = bj[j * stride];
                bj[j * stride] = bj[k * stride];
                bj[k * stride] = tmp;
            }
        } else {
            for (int j = 0; j < nw; j++) {
                int bnew = 0;
                bool dup = true;
                for (int guard = 0; dup && guard < 64; guard++) {
                    bnew = (int)r.below(U.modmax) + 2;
                    dup = false;
                    for (int k = 0; k < j; k++)
                        if (bj[k * stride] == bnew) dup = true;
                }
                bj[j * stride] = bnew;
            }
        }
        double sum = 0.0;
        for (int j = 0; j < nw; j++) {
            wj[j * stride] = -log(1.0 - r.f64());
            sum += wj[j * stride];
        }
        for (int j = 0; j < nw; j++) wj[j * stride] /= sum;
        for (int j = 0; j < nw; j++) {
            const int b = bj[j * stride];
            double amp = wj[j * stride] / (double)b;
            if (r.flip()) amp = -amp;
            if (b % 2 == 0) {
                const double f = r.f64() * kPi;
                double sf, cf;
                sincos(f, &sf, &cf);
                al[b * stride] += amp * cf;
                bt[b * stride] += amp * sf;
            } else {
                al[b * stride] += amp;
            }
        }
        a2[ax] = U.pin ? 0.0 : (r.f64() * 2.0 - 1.0);
    }
}

// FP64 position of one axis at timestep t from canonical coefficients: the
// contraction in ascending b (alpha_b S_bt, beta_b Cm_bt, alpha_b+1 S_b+1,t, ...),
// one fused multiply-add per term.  Table loads are issued four pairs ahead.
__device__ __forceinline__ double eval64(const UniDev& U, const double* alpha, const double* beta,
                                         int stride, double a2, int t) {
    const int T = U.T, F = U.F;
    const double* S = U.S + t;
    const double* Cm = U.Cm + t;
    double acc = 0.0;
    int b = 2;
#pragma unroll 4
    for (; b + 1 <= F; b += 2) {
        const double s0 = __ldg(S + (size_t)b * T), c0 = __ldg(Cm + (size_t)b * T);
        const double s1 = __ldg(S + (size_t)(b + 1) * T);
        acc = fma(alpha[b * stride], s0, acc);
        acc = fma(beta[b * stride], c0, acc);
        acc = fma(alpha[(b + 1) * stride], s1, acc);
    }
    if (b <= F) {  // even F: the last frequency has no odd partner
        acc = fma(alpha[b * stride], __ldg(S + (size_t)b * T), acc);
        acc = fma(beta[b * stride], __ldg(Cm + (size_t)b * T), acc);
    }
    return torus_wrap(fma(acc, __ldg(U.invsinz + t), a2));
}

// eval64 of D axes at once (coefficient rows ax * F1 of alpha / beta): each
// axis accumulates in eval64's order, so every coordinate has eval64's bits;
// the axes' chains are independent and the basis loads are shared.
template <int D>
__device__ __forceinline__ void eval64x(const UniDev& U, const double* alpha, const double* beta, const double* a2,
                                        int t, double* P) {
    const int T = U.T, F = U.F, F1 = F + 1;
    const double* S = U.S + t;
    const double* Cm = U.Cm + t;
    double acc[D];
#pragma unroll
    for (int ax = 0; ax < D; ax++) acc[ax] = 0.0;
    int b = 2;
#pragma unroll 2
    for (; b + 1 <= F; b += 2) {
        const double s0 = __ldg(S + (size_t)b * T), c0 = __ldg(Cm + (size_t)b * T);
        const double s1 = __ldg(S + (size_t)(b + 1) * T);
#pragma unroll
        for (int ax = 0; ax < D; ax++) {
            acc[ax] = fma(alpha[ax * F1 + b], s0, acc[ax]);
            acc[ax] = fma(beta[ax * F1 + b], c0, acc[ax]);
            acc[ax] = fma(alpha[ax * F1 + b + 1], s1, acc[ax]);
        }
    }
    if (b <= F) {
        const double s0 = __ldg(S + (size_t)b * T), c0 = __ldg(Cm + (size_t)b * T);
#pragma unroll
        for (int ax = 0; ax < D; ax++) {
            acc[ax] = fma(alpha[ax * F1 + b], s0, acc[ax]);
            acc[ax] = fma(beta[ax * F1 + b], c0, acc[ax]);
        }
    }
    const double iz = __ldg(U.invsinz + t);
#pragma unroll
    for (int ax = 0; ax < D; ax++) P[ax] = torus_wrap(fma(acc[ax], iz, a2[ax]));
}

// ------------------------------------------------------------ grid access

__device__ __forceinline__ uint64_t mix64(uint64_t k) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdULL;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ULL;
    k ^= k >> 33;
    return k;
}

// Loops over the axes run to the constant 3 (dim <= 3) so that callers' cell
// arrays stay in registers.
__device__ __forceinline__ int64_t lin_cell(const int* c, int dim, int gw) {
    int64_t lin = 0;
#pragma unroll
    for (int ax = 0; ax < 3; ax++)
        if (ax < dim) lin = lin * gw + c[ax];
    return lin;
}

// Head of the chain of accepted points in cell `lin` at timestep t (-1 none).
__device__ __forceinline__ int32_t grid_head(const UniDev& U, int t, int64_t lin, int64_t cells_per_t) {
    if (U.grid_kind == GRID_DENSE) return __ldg(U.heads + UG_IDX((int64_t)t * cells_per_t + lin, U.dense_cells));
    const uint64_t key = ((uint64_t)t << 40) | (uint64_t)lin;
    uint64_t h = mix64(key) & U.hmask;
    for (uint64_t probe = 0; probe <= U.hmask; probe++) {
        const ulonglong2 s = __ldg(U.hslot + UG_IDX(h, U.hmask + 1));  // key and head in one load
        if (s.x == key) return (int32_t)(uint32_t)s.y;
        if (s.x == kEmptyKey) return -1;
        h = (h + 1) & U.hmask;
    }
    return -1;
}

// Key of cell cc in the main grid and (coarse keys) the cell's bit in the slot's
// occupancy mask (0 for cell keys).
__device__ __forceinline__ int64_t grid_lin(const UniDev& U, const int* cc, uint32_t* fbit) {
    const int s = U.gkey_shift;
    if (s == 0) {
        *fbit = 0u;
        return lin_cell(cc, U.dim, U.gw);
    }
    int cs[3] = {0, 0, 0};
    uint32_t fi = 0;
#pragma unroll
    for (int ax = 0; ax < 3; ax++)
        if (ax < U.dim) {
            cs[ax] = cc[ax] >> s;
            fi = (fi << s) | (uint32_t)(cc[ax] & ((1 << s) - 1));
        }
    *fbit = 1u << fi;
    return lin_cell(cs, U.dim, U.occ_gw);
}

// Coarse-keyed grid: head of the chain of coarse cell `lin` at t and the mask of
// its occupied cells (0: no point).
__device__ __forceinline__ int32_t grid_head_mask(const UniDev& U, int t, int64_t lin, uint32_t* mask) {
    const uint64_t key = ((uint64_t)t << 40) | (uint64_t)lin;
    uint64_t h = mix64(key) & U.hmask;
    for (uint64_t probe = 0; probe <= U.hmask; probe++) {
        const ulonglong2 s = __ldg(U.hslot + UG_IDX(h, U.hmask + 1));
        if (s.x == key) {
            *mask = ~(uint32_t)(s.y >> 32);
            return (int32_t)(uint32_t)s.y;
        }
        if (s.x == kEmptyKey) break;
        h = (h + 1) & U.hmask;
    }
    *mask = 0u;
    return -1;
}

__device__ __forceinline__ int64_t cells_per_t(const UniDev& U) {
    int64_t n = 1;
#pragma unroll
    for (int ax = 0; ax < 3; ax++)
        if (ax < U.dim) n *= U.gw;
    return n;
}

// Bit of fine cell c at timestep t.  3+1: brick (c >> sh) >> 2, bit 16 r0 + 4 r1 + r2
// of its 64-bit word with r = (c >> sh) & 3; 2+1: brick (c >> sh) >> 3, bit 8 r0 + r1
// with r = (c >> sh) & 7; 1+1: coarse cells in a row.
__device__ __forceinline__ int64_t occ_bit(const UniDev& U, int t, const int* c) {
    if (U.dim == 2) {
        const int o0 = c[0] >> U.occ_shift, o1 = c[1] >> U.occ_shift;
        const int64_t brick = (int64_t)(o0 >> 3) * U.occ_nb + (o1 >> 3);
        return ((int64_t)t * U.occ_per_t + brick) * 64 + ((o0 & 7) << 3 | (o1 & 7));
    }
    if (U.dim == 3) {
        const int o0 = c[0] >> U.occ_shift, o1 = c[1] >> U.occ_shift, o2 = c[2] >> U.occ_shift;
        const int64_t brick = ((int64_t)(o0 >> 2) * U.occ_nb + (o1 >> 2)) * U.occ_nb + (o2 >> 2);
        return ((int64_t)t * U.occ_per_t + brick) * 64 + ((o0 & 3) << 4 | (o1 & 3) << 2 | (o2 & 3));
    }
    return (int64_t)t * U.occ_per_t + (c[0] >> U.occ_shift);  // dim 1
}
// Dilated filter: true when some committed point may lie within 2 cells of fine
// cell c at timestep t on every axis (false proves there is none).
template <int D>
__device__ __forceinline__ bool occ1_hit(const UniDev& U, int t, const int* c) {
    int64_t lin = 0;
#pragma unroll
    for (int ax = 0; ax < D; ax++) lin = lin * U.occ1_gw + (c[ax] >> U.occ1_shift);
    const int64_t b = (int64_t)t * U.occ1_per_t + lin;
    return (__ldg(U.occ1 + UG_IDX(b >> 5, U.occ1_words)) >> (b & 31)) & 1u;
}

__device__ __forceinline__ int wrap_cell(int v, int gw) {
    v += v < 0 ? gw : 0;
    return v >= gw ? v - gw : v;
}

// Neighbourhood of a point: per axis up to four wrapped cell coordinates
// (centre +-1, widened by one on a side when the point lies within the guard
// band of that cell face).  All loops below have constant trip counts and are
// fully unrolled; nothing divides.
template <int D>
struct Nbhd {
    int v[D][4];
    int n[D];
    int last[D];  // wrapped coordinate of the last cell per axis
};

template <int D>
__device__ __forceinline__ void nbhd_make(const UniDev& U, const int* c, const int* ext_lo,
                                          const int* ext_hi, Nbhd<D>& nb) {
#pragma unroll
    for (int ax = 0; ax < D; ax++) {
        const int lo = c[ax] - 1 - ext_lo[ax];
        nb.n[ax] = 3 + ext_lo[ax] + ext_hi[ax];
        nb.last[ax] = wrap_cell(c[ax] + 1 + ext_hi[ax], U.gw);
#pragma unroll
        for (int k = 0; k < 4; k++) nb.v[ax][k] = wrap_cell(lo + k, U.gw);
    }
}

// 4-bit mask x -> bits 4 i (i in x); and -> bits 16 i
__device__ __forceinline__ uint32_t spread4(uint32_t x) {
    return (x & 1u) | ((x & 2u) << 3) | ((x & 4u) << 6) | ((x & 8u) << 9);
}
__device__ __forceinline__ uint64_t spread16(uint32_t x) {
    return (uint64_t)(x & 1u) | ((uint64_t)(x & 2u) << 15) | ((uint64_t)(x & 4u) << 30) |
           ((uint64_t)(x & 8u) << 45);
}
__device__ __forceinline__ int cyc_dist(int f, int s, int gw) {  // (f - s) mod gw
    const int d = f - s;
    return d < 0 ? d + gw : d;
}

// Chains of the neighbourhood cells inside occupancy cell (o0, o1, o2) (3+1):
// the fine cells of that coarse cell that lie in the neighbourhood window of
// each axis (start nb.v[ax][0], nb.n[ax] cells, cyclic).
template <class Visit>
__device__ __forceinline__ bool brick_cell_visit(const UniDev& U, int t, const Nbhd<3>& nb, int64_t cpt, int o0,
                                              int o1, int o2, Visit& visit) {
    const int sh = U.occ_shift, gw = U.gw, w = 1 << sh;
    const int f0e = min(gw, (o0 + 1) * w), f1e = min(gw, (o1 + 1) * w), f2e = min(gw, (o2 + 1) * w);
    if (U.gkey_shift > 0) {  // one chain per coarse cell: walk it when a window cell is occupied
        uint32_t wm = 0u;
        for (int f0 = o0 * w; f0 < f0e; f0++) {
            if (cyc_dist(f0, nb.v[0][0], gw) >= nb.n[0]) continue;
            for (int f1 = o1 * w; f1 < f1e; f1++) {
                if (cyc_dist(f1, nb.v[1][0], gw) >= nb.n[1]) continue;
                for (int f2 = o2 * w; f2 < f2e; f2++)
                    if (cyc_dist(f2, nb.v[2][0], gw) < nb.n[2])
                        wm |= 1u << ((((f0 - o0 * w) << sh | (f1 - o1 * w)) << sh) | (f2 - o2 * w));
            }
        }
        uint32_t occm;
        const int oc[3] = {o0, o1, o2};
        int32_t p = grid_head_mask(U, t, lin_cell(oc, 3, U.occ_gw), &occm);
        if (!(occm & wm)) return false;
        while (p >= 0) {
            int32_t nx;
            if (visit(p, nx)) return true;
            p = nx;
        }
        return false;
    }
    for (int f0 = o0 * w; f0 < f0e; f0++) {
        if (cyc_dist(f0, nb.v[0][0], gw) >= nb.n[0]) continue;
        for (int f1 = o1 * w; f1 < f1e; f1++) {
            if (cyc_dist(f1, nb.v[1][0], gw) >= nb.n[1]) continue;
            for (int f2 = o2 * w; f2 < f2e; f2++) {
                if (cyc_dist(f2, nb.v[2][0], gw) >= nb.n[2]) continue;
                int32_t p = grid_head(U, t, ((int64_t)f0 * gw + f1) * gw + f2, cpt);
                while (p >= 0) {
                    int32_t nx;
                    if (visit(p, nx)) return true;
                    p = nx;
                }
            }
        }
    }
    return false;
}

// 3+1 neighbourhood scan over the brick layout.  Per axis the window's coarse
// cells fall into at most two bricks (a third only across the seam of a partial
// last brick: then every coarse cell is tested on its own).  Each brick
// combination costs one 64-bit word and a mask of the window's cells in it.
template <class Visit>
__device__ __forceinline__ bool nbhd_scan3(const UniDev& U, int t, const Nbhd<3>& nb, int64_t cpt,
                                           Visit&& visit) {
    const int sh = U.occ_shift, onb = U.occ_nb;
    int bA[3], bB[3];
    uint32_t mA[3], mB[3];
    bool three = false;
#pragma unroll
    for (int ax = 0; ax < 3; ax++) {
        const int oa = nb.v[ax][0] >> sh;
        bA[ax] = oa >> 2;
        bB[ax] = -1;
        mA[ax] = 1u << (oa & 3);
        mB[ax] = 0u;
#pragma unroll
        for (int k = 1; k < 4; k++) {
            if (k < nb.n[ax]) {
                const int o = nb.v[ax][k] >> sh, b = o >> 2;
                const uint32_t bit = 1u << (o & 3);
                if (b == bA[ax]) {
                    mA[ax] |= bit;
                } else if (bB[ax] < 0 || b == bB[ax]) {
                    bB[ax] = b;
                    mB[ax] |= bit;
                } else {
                    three = true;
                }
            }
        }
    }
    const int64_t tb = (int64_t)t * U.occ_per_t;
    const uint64_t* W = reinterpret_cast<const uint64_t*>(U.occ);
    if (!three) {
        uint64_t hits[8];
#pragma unroll
        for (int c = 0; c < 8; c++) {
            const int B0 = (c & 4) ? bB[0] : bA[0], B1 = (c & 2) ? bB[1] : bA[1], B2 = (c & 1) ? bB[2] : bA[2];
            hits[c] = 0;
            if (B0 < 0 || B1 < 0 || B2 < 0) continue;
            const uint32_t M0 = (c & 4) ? mB[0] : mA[0], M1 = (c & 2) ? mB[1] : mA[1], M2 = (c & 1) ? mB[2] : mA[2];
            const uint64_t m = (uint64_t)(M2 * spread4(M1)) * spread16(M0);
            hits[c] = __ldg(W + UG_IDX(tb + ((int64_t)B0 * onb + B1) * onb + B2, U.occ_words / 2)) & m;
        }
        uint32_t pend = 0;
#pragma unroll
        for (int c = 0; c < 8; c++) pend |= hits[c] ? 1u << c : 0u;
        while (pend) {
            const int c = __ffs(pend) - 1;
            pend &= pend - 1;
            uint64_t h = hits[0];
#pragma unroll
            for (int q = 1; q < 8; q++)
                if (q == c) h = hits[q];
            const int B0 = (c & 4) ? bB[0] : bA[0], B1 = (c & 2) ? bB[1] : bA[1], B2 = (c & 1) ? bB[2] : bA[2];
            while (h) {
                const int bit = __ffsll((long long)h) - 1;
                h &= h - 1;
                if (brick_cell_visit(U, t, nb, cpt, B0 * 4 + (bit >> 4), B1 * 4 + ((bit >> 2) & 3),
                                     B2 * 4 + (bit & 3), visit))
                    return true;
            }
        }
        return false;
    }
    // rare: a third brick on some axis -- test every coarse cell of the window
    for (int k0 = 0; k0 < nb.n[0]; k0++) {
        const int f0 = nb.v[0][0] + k0 >= U.gw ? nb.v[0][0] + k0 - U.gw : nb.v[0][0] + k0;
        if (k0 > 0 && (f0 >> sh) == ((f0 == 0 ? U.gw - 1 : f0 - 1) >> sh)) continue;  // same coarse cell
        for (int k1 = 0; k1 < nb.n[1]; k1++) {
            const int f1 = nb.v[1][0] + k1 >= U.gw ? nb.v[1][0] + k1 - U.gw : nb.v[1][0] + k1;
            if (k1 > 0 && (f1 >> sh) == ((f1 == 0 ? U.gw - 1 : f1 - 1) >> sh)) continue;
            for (int k2 = 0; k2 < nb.n[2]; k2++) {
                const int f2 = nb.v[2][0] + k2 >= U.gw ? nb.v[2][0] + k2 - U.gw : nb.v[2][0] + k2;
                if (k2 > 0 && (f2 >> sh) == ((f2 == 0 ? U.gw - 1 : f2 - 1) >> sh)) continue;
                const int cc[3] = {f0, f1, f2};
                const int64_t b = occ_bit(U, t, cc);
                if (!((__ldg(U.occ + UG_IDX(b >> 5, U.occ_words)) >> (b & 31)) & 1u)) continue;
                if (brick_cell_visit(U, t, nb, cpt, f0 >> sh, f1 >> sh, f2 >> sh, visit)) return true;
            }
        }
    }
    return false;
}

// 1+1: coarse cells along the words.
template <int D, class Visit>
__device__ __forceinline__ bool nbhd_scan_rows(const UniDev& U, int t, const Nbhd<D>& nb, int64_t cpt,
                                               Visit&& visit) {
    const int gw = U.gw, sh = U.occ_shift, ogw = U.occ_gw;
    const int64_t tb = (int64_t)t * U.occ_per_t;
    constexpr int L = D - 1;  // the last axis runs along the bitmap words
    const int nl = nb.n[L];
#pragma unroll
    for (int i0 = 0; i0 < (D > 1 ? 4 : 1); i0++) {
        if (D > 1 && i0 >= nb.n[0]) break;
#pragma unroll
        for (int i1 = 0; i1 < (D > 2 ? 4 : 1); i1++) {
            if (D > 2 && i1 >= nb.n[D > 2 ? 1 : 0]) break;
            int64_t orow = 0, lrow = 0;  // row prefixes: bitmap (coarse) and grid (fine)
            if (D > 1) {
                const int x0 = nb.v[0][i0];
                orow = x0 >> sh;
                lrow = x0;
            }
            if (D > 2) {
                const int x1 = nb.v[D > 2 ? 1 : 0][i1];
                orow = orow * ogw + (x1 >> sh);
                lrow = lrow * gw + x1;
            }
            const int64_t obase = tb + orow * ogw;
            // the row's cells lie in the words of its first and last cell
            const int64_t bf = obase + (nb.v[L][0] >> sh), bl = obase + (nb.last[L] >> sh);
            const uint32_t wf = __ldg(U.occ + UG_IDX(bf >> 5, U.occ_words));
            const uint32_t wl = (bl >> 5) == (bf >> 5) ? wf : __ldg(U.occ + UG_IDX(bl >> 5, U.occ_words));
            uint32_t row_bits = 0;
#pragma unroll
            for (int k = 0; k < 4; k++) {
                if (k >= nl) break;
                const int64_t bk = obase + (nb.v[L][k] >> sh);
                uint32_t w;
                if ((bk >> 5) == (bf >> 5))
                    w = wf;
                else if ((bk >> 5) == (bl >> 5))
                    w = wl;
                else
                    w = __ldg(U.occ + UG_IDX(bk >> 5, U.occ_words));
                row_bits |= ((w >> (bk & 31)) & 1u) << k;
            }
            while (row_bits) {
                const int k = __ffs(row_bits) - 1;
                row_bits &= row_bits - 1;
                int xl = nb.v[L][0];
#pragma unroll
                for (int q = 1; q < 4; q++)
                    if (q == k) xl = nb.v[L][q];
                const int64_t lin = D > 1 ? lrow * gw + xl : (int64_t)xl;
                int32_t p = grid_head(U, t, lin, cpt);
                while (p >= 0) {
                    int32_t nx;
                    if (visit(p, nx)) return true;
                    p = nx;
                }
            }
        }
    }
    return false;
}

// 8-bit mask x -> bits 8 i (i in x)
__device__ __forceinline__ uint64_t spread8(uint32_t x) {
    uint64_t r = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) r |= (uint64_t)((x >> i) & 1u) << (8 * i);
    return r;
}

// 2+1 counterpart of brick_cell_visit.
template <class Visit>
__device__ __forceinline__ bool brick_cell_visit2(const UniDev& U, int t, const Nbhd<2>& nb, int64_t cpt, int o0,
                                                  int o1, Visit& visit) {
    const int sh = U.occ_shift, gw = U.gw, w = 1 << sh;
    const int f0e = min(gw, (o0 + 1) * w), f1e = min(gw, (o1 + 1) * w);
    if (U.gkey_shift > 0) {  // one chain per coarse cell: walk it when a window cell is occupied
        uint32_t wm = 0u;
        for (int f0 = o0 * w; f0 < f0e; f0++) {
            if (cyc_dist(f0, nb.v[0][0], gw) >= nb.n[0]) continue;
            for (int f1 = o1 * w; f1 < f1e; f1++)
                if (cyc_dist(f1, nb.v[1][0], gw) < nb.n[1]) wm |= 1u << ((f0 - o0 * w) << sh | (f1 - o1 * w));
        }
        uint32_t occm;
        const int oc[2] = {o0, o1};
        int32_t p = grid_head_mask(U, t, lin_cell(oc, 2, U.occ_gw), &occm);
        if (!(occm & wm)) return false;
        while (p >= 0) {
            int32_t nx;
            if (visit(p, nx)) return true;
            p = nx;
        }
        return false;
    }
    for (int f0 = o0 * w; f0 < f0e; f0++) {
        if (cyc_dist(f0, nb.v[0][0], gw) >= nb.n[0]) continue;
        for (int f1 = o1 * w; f1 < f1e; f1++) {
            if (cyc_dist(f1, nb.v[1][0], gw) >= nb.n[1]) continue;
            int32_t p = grid_head(U, t, (int64_t)f0 * gw + f1, cpt);
            while (p >= 0) {
                int32_t nx;
                if (visit(p, nx)) return true;
                p = nx;
            }
        }
    }
    return false;
}

// 2+1 neighbourhood scan over 8x8 bricks (as nbhd_scan3: at most two bricks per
// axis, a third only across the seam of a partial last brick).
template <class Visit>
__device__ __forceinline__ bool nbhd_scan2(const UniDev& U, int t, const Nbhd<2>& nb, int64_t cpt,
                                           Visit&& visit) {
    const int sh = U.occ_shift, onb = U.occ_nb;
    int bA[2], bB[2];
    uint32_t mA[2], mB[2];
    bool three = false;
#pragma unroll
    for (int ax = 0; ax < 2; ax++) {
        const int oa = nb.v[ax][0] >> sh;
        bA[ax] = oa >> 3;
        bB[ax] = -1;
        mA[ax] = 1u << (oa & 7);
        mB[ax] = 0u;
#pragma unroll
        for (int k = 1; k < 4; k++) {
            if (k < nb.n[ax]) {
                const int o = nb.v[ax][k] >> sh, b = o >> 3;
                const uint32_t bit = 1u << (o & 7);
                if (b == bA[ax]) {
                    mA[ax] |= bit;
                } else if (bB[ax] < 0 || b == bB[ax]) {
                    bB[ax] = b;
                    mB[ax] |= bit;
                } else {
                    three = true;
                }
            }
        }
    }
    const int64_t tb = (int64_t)t * U.occ_per_t;
    const uint64_t* W = reinterpret_cast<const uint64_t*>(U.occ);
    if (!three) {
        uint64_t hits[4];
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int B0 = (c & 2) ? bB[0] : bA[0], B1 = (c & 1) ? bB[1] : bA[1];
            hits[c] = 0;
            if (B0 < 0 || B1 < 0) continue;
            const uint32_t M0 = (c & 2) ? mB[0] : mA[0], M1 = (c & 1) ? mB[1] : mA[1];
            hits[c] = __ldg(W + UG_IDX(tb + (int64_t)B0 * onb + B1, U.occ_words / 2)) & ((uint64_t)M1 * spread8(M0));
        }
        uint32_t pend = 0;
#pragma unroll
        for (int c = 0; c < 4; c++) pend |= hits[c] ? 1u << c : 0u;
        while (pend) {
            const int c = __ffs(pend) - 1;
            pend &= pend - 1;
            uint64_t h = hits[0];
#pragma unroll
            for (int q = 1; q < 4; q++)
                if (q == c) h = hits[q];
            const int B0 = (c & 2) ? bB[0] : bA[0], B1 = (c & 1) ? bB[1] : bA[1];
            while (h) {
                const int bit = __ffsll((long long)h) - 1;
                h &= h - 1;
                if (brick_cell_visit2(U, t, nb, cpt, B0 * 8 + (bit >> 3), B1 * 8 + (bit & 7), visit)) return true;
            }
        }
        return false;
    }
    for (int k0 = 0; k0 < nb.n[0]; k0++) {
        const int f0 = nb.v[0][0] + k0 >= U.gw ? nb.v[0][0] + k0 - U.gw : nb.v[0][0] + k0;
        if (k0 > 0 && (f0 >> sh) == ((f0 == 0 ? U.gw - 1 : f0 - 1) >> sh)) continue;
        for (int k1 = 0; k1 < nb.n[1]; k1++) {
            const int f1 = nb.v[1][0] + k1 >= U.gw ? nb.v[1][0] + k1 - U.gw : nb.v[1][0] + k1;
            if (k1 > 0 && (f1 >> sh) == ((f1 == 0 ? U.gw - 1 : f1 - 1) >> sh)) continue;
            const int cc[2] = {f0, f1};
            const int64_t b = occ_bit(U, t, cc);
            if (!((__ldg(U.occ + UG_IDX(b >> 5, U.occ_words)) >> (b & 31)) & 1u)) continue;
            if (brick_cell_visit2(U, t, nb, cpt, f0 >> sh, f1 >> sh, visit)) return true;
        }
    }
    return false;
}

// Visit the chains of the occupied cells of the neighbourhood at timestep t.
// visit(p) returns true to stop (the scan then returns true).
template <int D, class Visit>
__device__ __forceinline__ bool nbhd_scan(const UniDev& U, int t, const Nbhd<D>& nb, int64_t cpt,
                                          Visit&& visit) {
    if constexpr (D == 3) {
        return nbhd_scan3(U, t, nb, cpt, visit);
    } else if constexpr (D == 2) {
        return nbhd_scan2(U, t, nb, cpt, visit);
    } else {
        return nbhd_scan_rows<D>(U, t, nb, cpt, visit);
    }
}


// Contacts of the point P at timestep t with the accepted packing (FP64,
// exact): the neighbourhood is the centre cell +-1 on every axis.  Unique
// mode: true on the first contact.  Group mode: accumulates the single
// touched group in *g and returns true when a second distinct group appears.
template <int D>
__device__ __forceinline__ bool contacts64_d(const UniDev& U, int t, const double* P, bool group,
                                             int32_t* g, int64_t cpt, int* nvis) {
    int c[D], z[D];
#pragma unroll
    for (int ax = 0; ax < D; ax++) {
        c[ax] = cell_of(P[ax], U.cell, U.gw);
        z[ax] = 0;
    }
    if (!occ1_hit<D>(U, t, c)) return false;
    Nbhd<D> nb;
    nbhd_make<D>(U, c, z, z, nb);
    return nbhd_scan<D>(U, t, nb, cpt, [&](int32_t p, int32_t& nx) -> bool {
        const Pt64* q = U.pts + UG_IDX((int64_t)p * U.T + t, U.slot_cap * U.T);
        nx = __ldg(&q->next);
        if (nvis) ++*nvis;
        double Q[3];
#pragma unroll
        for (int ax = 0; ax < D; ax++) Q[ax] = __ldg(&q->c[ax]);
        if (U.gkey_shift > 0) {  // coarse chains: only the points of the 3^D window cells count
#pragma unroll
            for (int ax = 0; ax < D; ax++)
                if (cyc_dist(cell_of(Q[ax], U.cell, U.gw), nb.v[ax][0], U.gw) >= nb.n[ax]) return false;
        }
        if (!pair_hit64(U, P, Q)) return false;
        if (!group) return true;
        const int32_t gq = __ldg(&q->gid);
        if (*g == -1) {
            *g = gq;
            return false;
        }
        return *g != gq;
    });
}

__device__ __forceinline__ bool contacts64(const UniDev& U, int t, const double* P, bool group,
                                           int32_t* g, int64_t cpt, int* nvis = nullptr) {
    if (U.dim == 3) return contacts64_d<3>(U, t, P, group, g, cpt, nvis);
    if (U.dim == 2) return contacts64_d<2>(U, t, P, group, g, cpt, nvis);
    return contacts64_d<1>(U, t, P, group, g, cpt, nvis);
}

// 1+1D crossing rule: minimum-image separation changes sign between
// consecutive timesteps with |d_t| + |d_t+1| < 1.  No reference counterpart.
__device__ __forceinline__ bool crosses_step(double d0, double d1) {
    return ((d0 < 0.0) != (d1 < 0.0)) && fabs(d0) + fabs(d1) < 1.0;
}

}  // namespace ug
