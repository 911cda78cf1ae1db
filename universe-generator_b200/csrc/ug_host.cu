// ug_host.cu -- host runtime and C ABI of the packer (include/ug.h).
//
// One handle = one batch of independent universes on one GPU.  The host
// allocates every universe's tables, grid, point store and round buffers,
// then replays the round pipeline (ug_kernels.cu) -- optionally captured as
// a CUDA graph of `rounds_per_sync` rounds -- and reads back the small
// control blocks between replays to grow capacities and detect completion.
// Nothing per candidate crosses PCIe.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/ug.h"
#include "ug_frames.cuh"
#include "ug_kernels.cuh"
#include "ug_mixed.cuh"

namespace ug {

#ifdef UG_CHECKED
__device__ unsigned long long ug_check_record[4];
#endif

static thread_local std::string g_err;

static int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define CKR(x)                                                                                \
    do {                                                                                      \
        cudaError_t e_ = (x);                                                                 \
        if (e_ != cudaSuccess)                                                                \
            return fail(e_ == cudaErrorMemoryAllocation ? UG_ENOMEM : UG_ECUDA, "%s:%d %s: %s", \
                        __FILE__, __LINE__, #x, cudaGetErrorString(e_));                      \
    } while (0)

enum KernelId {
    K_PLAN, K_PRE, K_MIXED, K_CONFIRM, K_COMPACT, K_SGEN, K_CONFL, K_GREEDY, K_COMMIT, K_SGEMM, K_SHASH,
    K_NK
};
static const char* kKernelNames[12] = {"k_plan",      "k_prefilter64w", "k_prefilter_mixed",
                                       "k_confirm64w", "k_compact",     "k_surv_gen",
                                       "k_conflicts", "k_greedy",      "k_commit",
                                       "k_surv_gemm", "k_surv_hash",   ""};

struct UniHost {
    ug_universe_cfg cfg;
    UniDev d;
    std::vector<void*> owned;  // fixed-size allocations
    int64_t dense_bytes = 0;
    int64_t hcap = 0;
    int64_t occ_words = 0, occ1_words = 0;
    MixedTables mt;            // tensor-core operand tables (mixed precision)
};

struct Batch {
    int dev = 0;
    cudaStream_t st = nullptr;
    bool own_stream = false;
    int n = 0;
    int nsm = 148;
    ug_run_opts opts{};
    std::vector<UniHost> U;
    UniDev* dU = nullptr;
    UniCtl* dCtl = nullptr;
    std::vector<UniCtl> hCtl;
    RoundInfo* dInfo = nullptr;
    cudaGraphExec_t gexec = nullptr;
    int graph_rounds = 0;
    cudaEvent_t ev[2 * K_NK]{};
    double kms[K_NK]{};
    int64_t klaunch[K_NK]{};
    bool synced = false;
    int max_T = 0;
    bool any_mixed = false;
    bool any_group = false;   // some universe runs group rounds
    bool any_euclid = false;  // some universe excludes by the L2 ball
    bool any_knot = false;    // some universe draws from the knot stream
    int64_t launches = 0;  // kernels issued (graph replays count every node)
    int64_t h2d = 0, d2h = 0;  // bytes copied between host and device
    int kernels_per_round = 9;
    // CTAs per SM of grid-stride round kernels sized from the occupancy at creation
    int res_sgen = 8, res_shash = 8, res_confl = 16;
    // bulk read-back staging (ug_batch_accepted_all)
    int64_t* d_gather_idx = nullptr;
    int32_t* d_gather_gid = nullptr;
    int64_t* d_gather_off = nullptr;
    int64_t gather_cap = 0;
};

// CTAs per SM a grid-stride kernel is launched with: at most as many as can be
// resident, so that its static item striding runs in one wave (a CTA beyond that
// starts only when a resident one has finished all of its items).
template <class F>
static int resident_ctas(F* fn, int threads, size_t smem, int cap) {
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, threads, smem) != cudaSuccess || nb < 1) {
        cudaGetLastError();
        return 1;
    }
    return std::min(nb, cap);
}

static int64_t pow2_at_least(int64_t v) {
    int64_t p = 1;
    while (p < v) p <<= 1;
    return p;
}

template <class T>
static int dalloc(UniHost& h, T** p, size_t n, int fill = -2) {
    void* q = nullptr;
    if (n == 0) n = 1;
    CKR(cudaMalloc(&q, n * sizeof(T)));
    if (fill != -2) CKR(cudaMemset(q, fill, n * sizeof(T)));
    h.owned.push_back(q);
    *p = (T*)q;
    return UG_OK;
}

static int validate(const ug_universe_cfg& c) {
    if (c.dim < 1 || c.dim > 3) return fail(UG_EINVAL, "dim must be 1, 2 or 3 (got %d)", c.dim);
    if (c.T < 4 || c.T > kMaxF) return fail(UG_EINVAL, "T must be in [4, %d] (got %d)", kMaxF, c.T);
    const int terms = c.terms ? c.terms : c.T;
    const int modmax = c.T - 1 > 2 ? c.T - 1 : 2;
    if (terms < 2 || terms - 1 > modmax)
        return fail(UG_EINVAL, "--terms %d exceeds unique-frequency pool %d (max terms %d)", terms,
                    modmax, modmax + 1);
    if (c.rng == UG_RNG_PHILOX && terms != c.T)
        return fail(UG_EINVAL, "the Philox stream is full band only (terms must be T)");
    if (c.rng != UG_RNG_PHILOX && c.rng != UG_RNG_KNOT) return fail(UG_EINVAL, "bad rng %d", c.rng);
    if (c.zgrid != UG_ZGRID_REF && c.zgrid != UG_ZGRID_MID) return fail(UG_EINVAL, "bad zgrid");
    if (c.excl != UG_EXCL_REF && c.excl != UG_EXCL_OPEN) return fail(UG_EINVAL, "bad excl");
    if (c.group_mode < 0 || c.group_mode > 2) return fail(UG_EINVAL, "bad group_mode");
    if (c.attempts < 0 || c.max_n < 0 || c.sub_attempts < 0) return fail(UG_EINVAL, "negative budget");
    if (c.round_size < 0 || c.round_size > (1 << 20) || (c.round_size % kTile))
        return fail(UG_EINVAL, "round_size must be a multiple of %d up to 2^20", kTile);
    if (c.surv_cap < 0 || c.surv_cap > kSmaxCap || (c.surv_cap % 32))
        return fail(UG_EINVAL, "surv_cap must be a multiple of 32 up to %d", (int)kSmaxCap);
    if (c.cross1d && c.dim != 1) return fail(UG_EINVAL, "cross1d applies to dim 1 only");
    if (c.euclid != 0 && c.euclid != 1) return fail(UG_EINVAL, "bad euclid flag");
    return UG_OK;
}

// Host FP64 tables: z grid, 1/sin z, sin(b z), cos(b z) - 1, endpoint-first order.
static void host_tables(const ug_universe_cfg& c, std::vector<double>& S, std::vector<double>& Cm,
                        std::vector<double>& inv, std::vector<int32_t>& order) {
    const int T = c.T, F = c.T;
    std::vector<double> z(T);
    inv.resize(T);
    for (int i = 0; i < T; i++) {
        z[i] = c.zgrid == UG_ZGRID_REF ? (i + 1) * kPi / (T + 1) : (i + 0.5) * kPi / T;
        inv[i] = 1.0 / sin(z[i]);
    }
    S.assign((size_t)(F + 1) * T, 0.0);
    Cm.assign((size_t)(F + 1) * T, 0.0);
    for (int b = 0; b <= F; b++)
        for (int t = 0; t < T; t++) {
            S[(size_t)b * T + t] = sin(b * z[t]);
            Cm[(size_t)b * T + t] = cos(b * z[t]) - 1.0;
        }
    order.resize(T);
    for (int i = 0; i < T; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return std::min(a, T - 1 - a) < std::min(b, T - 1 - b);
    });
}

static int alloc_points(UniHost& h, int64_t cap) {
    const int T = h.cfg.T;
    Pt64* p = nullptr;
    Pt32* f = nullptr;
    int64_t* ai = nullptr;
    CKR(cudaMalloc(&p, (size_t)cap * T * sizeof(Pt64)));
    CKR(cudaMalloc(&f, (size_t)cap * T * sizeof(Pt32)));
    CKR(cudaMalloc(&ai, (size_t)cap * sizeof(int64_t)));
    h.d.pts = p;
    h.d.ptf = f;
    h.d.acc_idx = ai;
    h.d.slot_cap = cap;
    return UG_OK;
}

// Hash grid of cap slots, all empty (key and head all ones: no key, head -1).
static int alloc_hash(UniHost& h, int64_t cap) {
    ulonglong2* s = nullptr;
    CKR(cudaMalloc(&s, (size_t)cap * sizeof(ulonglong2)));
    CKR(cudaMemset(s, 0xff, (size_t)cap * sizeof(ulonglong2)));
    h.d.hslot = s;
    h.d.hmask = (uint64_t)(cap - 1);
    h.hcap = cap;
    return UG_OK;
}

static int setup_universe(Batch& B, UniHost& h, int64_t dense_budget, int64_t* dense_used) {
    const ug_universe_cfg& c = h.cfg;
    UniDev& d = h.d;
    memset(&d, 0, sizeof d);
    d.dim = c.dim;
    d.T = c.T;
    d.F = c.T;
    d.nw = (c.terms ? c.terms : c.T) - 1;
    d.rng = c.rng;
    d.cross1d = c.cross1d;
    d.euclid = c.euclid;
    d.pin = c.pin_sin1;
    d.group_mode = c.group_mode;
    d.seed = c.seed;
    d.modmax = (uint32_t)(c.T - 1 > 2 ? c.T - 1 : 2);
    if (c.excl == UG_EXCL_REF) {
        d.cell = 2.0 / c.T;
        d.gw = c.T;
        d.inclusive = 1;
    } else {
        d.cell = 1.0 / c.T;
        d.gw = 2 * c.T;
        d.inclusive = 0;
    }
    d.B_max = c.round_size ? c.round_size : 65536;
    const int T = c.T;
    d.S_max = (int)std::min<int64_t>(kSmaxCap, std::max<int64_t>(256, (1 << 20) / T));
    if (c.dim == 1) d.S_max = 256;  // 1+1D in-round conflicts are found pairwise
    // Round-table block of 2^s cells per axis: a survivor timestep probes the blocks
    // of its 3-cell window (2 per axis at s = 1, 1 + 2 / 2^s on average above) and
    // walks their chains (2^(s dim) cells of at most S_max / gw^dim points each).
    // The block minimising probes * (1 + expected chain points) is taken: sparse
    // universes (large F) get large blocks, crowded ones 2 cells (c3 with the direct
    // table: 366.0 ms of kernels against 369.5 / 370.3 ms with chain points weighted
    // 2 / 4).
    {
        const double rho = (double)d.S_max / std::pow((double)d.gw, (double)c.dim);
        double best = 1e300;
        for (int sh = 1; sh <= 4; sh++) {
            const double w = (double)(1 << sh);
            const double probes = std::pow(sh == 1 ? 2.0 : 1.0 + 2.0 / w, (double)c.dim);
            const double cost = probes * (1.0 + std::pow(w, (double)c.dim) * rho);
            if (cost < best) {
                best = cost;
                d.rblock_shift = sh;
            }
        }
    }
    if (c.surv_cap > 0) d.S_max = c.surv_cap;
    d.S_max = std::min(d.S_max, d.B_max);
    // tables
    std::vector<double> S, Cm, inv;
    std::vector<int32_t> order;
    host_tables(c, S, Cm, inv, order);
    double *dS, *dC, *dI;
    int32_t* dO;
    int rc;
    if ((rc = dalloc(h, &dS, S.size())) || (rc = dalloc(h, &dC, Cm.size())) ||
        (rc = dalloc(h, &dI, inv.size())) || (rc = dalloc(h, &dO, order.size())))
        return rc;
    CKR(cudaMemcpy(dS, S.data(), S.size() * 8, cudaMemcpyHostToDevice));
    CKR(cudaMemcpy(dC, Cm.data(), Cm.size() * 8, cudaMemcpyHostToDevice));
    CKR(cudaMemcpy(dI, inv.data(), inv.size() * 8, cudaMemcpyHostToDevice));
    CKR(cudaMemcpy(dO, order.data(), order.size() * 4, cudaMemcpyHostToDevice));
    d.S = dS;
    d.Cm = dC;
    d.invsinz = dI;
    d.order = dO;
    // term-ordered table of the survivor product (row kseq_s(b): sin(b z),
    // row kseq_s(b) + 1 for even b: cos(b z) - 1), timesteps padded to 32
    {
        const int F = d.F;
        d.K = kseq_len(F);
        d.Tpad = (T + 31) / 32 * 32;
        d.Rpad = (d.S_max * c.dim + 31) / 32 * 32;
        std::vector<double> kt((size_t)d.K * d.Tpad, 0.0);
        for (int b = 2; b <= F; b++) {
            const int k = kseq_s(b);
            for (int t = 0; t < T; t++) {
                kt[(size_t)k * d.Tpad + t] = S[(size_t)b * T + t];
                if (!(b & 1)) kt[(size_t)(k + 1) * d.Tpad + t] = Cm[(size_t)b * T + t];
            }
        }
        double* dK;
        if ((rc = dalloc(h, &dK, kt.size())) || (rc = dalloc(h, &d.coef, (size_t)d.K * d.Rpad, 0)) ||
            (rc = dalloc(h, &d.a2row, (size_t)d.Rpad, 0)))
            return rc;
        CKR(cudaMemcpy(dK, kt.data(), kt.size() * 8, cudaMemcpyHostToDevice));
        d.KT = dK;
    }
    // grid
    int64_t cpt = 1;
    for (int ax = 0; ax < c.dim; ax++) cpt *= d.gw;
    const int64_t dense = (int64_t)T * cpt * 4;
    if (!B.opts.force_hash && dense <= (int64_t)4 << 30 && *dense_used + dense <= dense_budget) {
        d.grid_kind = GRID_DENSE;
        if ((rc = dalloc(h, &d.heads, (size_t)T * cpt, 0xff))) return rc;
        d.dense_cells = (int64_t)T * cpt;
        h.dense_bytes = dense;
        *dense_used += dense;
    } else {
        d.grid_kind = GRID_HASH;
        if ((rc = alloc_hash(h, pow2_at_least(std::max<int64_t>(1 << 16, 4LL * d.S_max * T)))))
            return rc;
    }
    // occupancy bitmap, coarsened until it is at most 512 MiB (T <= 256 in 3D
    // keeps 2 cells per coarse cell per axis or finer)
    {
        int sh = 0;
        int64_t bits;
        for (;; sh++) {
            const int64_t g = (d.gw + (1 << sh) - 1) >> sh;
            int64_t per = 1;
            if (c.dim == 3) {  // 4x4x4 bricks of 64 bits
                const int64_t nbk = (g + 3) >> 2;
                per = nbk * nbk * nbk;
                bits = (int64_t)T * per * 64;
                d.occ_nb = (int32_t)nbk;
            } else if (c.dim == 2) {  // 8x8 bricks of 64 bits
                const int64_t nbk = (g + 7) >> 3;
                per = nbk * nbk;
                bits = (int64_t)T * per * 64;
                d.occ_nb = (int32_t)nbk;
            } else {
                for (int ax = 0; ax < c.dim; ax++) per *= g;
                bits = (int64_t)T * per;
            }
            if (bits <= ((int64_t)1 << 32) || sh >= 4) {
                d.occ_shift = sh;
                d.occ_gw = (int32_t)g;
                d.occ_per_t = per;
                break;
            }
        }
        h.occ_words = (bits + 31) / 32;
        d.occ_words = h.occ_words;
        // A coarsened bitmap leaves several cells per occupied bit; the hash grid then
        // keys the coarse cells too (one probe per occupied coarse cell instead of
        // one per window cell in it), with the cells' occupancy mask in the slot.
        d.gkey_shift = (d.grid_kind == GRID_HASH && c.dim >= 2 && sh * c.dim <= 5) ? sh : 0;
        if ((rc = dalloc(h, &d.occ, (size_t)h.occ_words, 0))) return rc;
        // the finest blocks within 16 MiB (2^27 bits): commits mark it at random and
        // every test reads it, so a small map that stays in L2 pays more than fine
        // blocks (c3 job: 2^27 bits 513 ms, 2^29 515 ms, 2^32 541 ms).  The FP64
        // path needs the radius alone (the tensor-core setup widens it by the band)
        d.occ1_reach = d.cell * 1.001;
        int64_t per1 = 1;
        for (int s1 = 0;; s1++) {
            d.occ1_shift = s1;
            d.occ1_gw = (d.gw + (1 << s1) - 1) >> s1;
            per1 = 1;
            for (int ax = 0; ax < c.dim; ax++) per1 *= d.occ1_gw;
            if ((int64_t)T * per1 <= ((int64_t)1 << 27) || s1 >= 6) break;
        }
        d.occ1_per_t = per1;
        h.occ1_words = ((int64_t)T * per1 + 31) / 32;
        d.occ1_words = h.occ1_words;
        if ((rc = dalloc(h, &d.occ1, (size_t)h.occ1_words, 0))) return rc;
    }
    // accepted points
    const int64_t total_budget =
        c.attempts + (c.group_mode == UG_GROUP_SUBPATH ? (c.sub_attempts ? c.sub_attempts : c.attempts) : 0);
    int64_t cap = B.opts.slot_hint > 0 ? B.opts.slot_hint : 8192;
    cap = std::max<int64_t>(std::min<int64_t>(cap, total_budget + 1), 1024);
    if ((rc = alloc_points(h, cap))) return rc;
    // round buffers
    const int Bm = d.B_max, Sm = d.S_max;
    if ((rc = dalloc(h, &d.surv_bits, Bm / 32, 0)) || (rc = dalloc(h, &d.gray_bits, Bm / 32, 0)) ||
        (rc = dalloc(h, &d.gray_off, Bm, 0)) ||
        (rc = dalloc(h, &d.g0, Bm, 0xff)) || (rc = dalloc(h, &d.surv_off, Sm + 1, 0)) ||
        (rc = dalloc(h, &d.spos, (size_t)Sm * T, 0)) || (rc = dalloc(h, &d.ccount, Sm, 0)) ||
        (rc = dalloc(h, &d.clist, (size_t)Sm * kConflictCap, 0)) ||
        (rc = dalloc(h, &d.sgid, Sm, 0xff)) || (rc = dalloc(h, &d.acc_rank, Sm, 0xff)))
        return rc;
    // Round table: one 8-byte head per (timestep, block), at most 2^25 entries (the
    // block grows past the cost model's choice if needed).
    for (;; d.rblock_shift++) {
        const int64_t g = (d.gw + (1 << d.rblock_shift) - 1) >> d.rblock_shift;
        d.rblocks = 1;
        for (int ax = 0; ax < c.dim; ax++) d.rblocks *= g;
        if ((int64_t)T * d.rblocks <= ((int64_t)1 << 25) || d.rblock_shift >= 6) break;
    }
    if ((rc = dalloc(h, &d.rhead, (size_t)T * d.rblocks, 0xff))) return rc;
    return UG_OK;
}

static void init_ctl(const ug_universe_cfg& c, const UniDev& d, UniCtl& k) {
    memset(&k, 0, sizeof k);
    k.next_cand = 0;
    k.phase_end = c.attempts;
    k.sub_budget = c.sub_attempts ? c.sub_attempts : c.attempts;
    k.max_n = c.max_n;
    k.phase = 1;
    k.state = ST_ACTIVE;
    k.B_min = std::min(1024, d.B_max);
    k.B_cap = d.B_max;
    // first round: at most half a timestep's cells (a small torus jams after few
    // paths, and a round far above that only piles up in-round conflicts);
    // adapted every round after that
    int64_t cpt = 1;
    for (int ax = 0; ax < c.dim; ax++) cpt *= d.gw;
    int64_t b0 = std::max(4096, 2 * d.S_max);
    if (cpt / 2 < b0) b0 = std::max<int64_t>(1024, cpt / 2);
    k.round_B = (int)std::min<int64_t>(b0, d.B_max) / kTile * kTile;
    k.accept_rate = c.accept_rate;
    k.sub_accept_rate = c.sub_accept_rate;
    k.win_thr = c.accept_rate;
    k.win_q = win_bucket(c.accept_rate);
    k.sub_fill_rate = c.sub_fill_rate;
    k.fwin_q = 0;  // armed when phase 2 starts
}

static int push_unidev(Batch& B) {
    std::vector<UniDev> v(B.n);
    for (int i = 0; i < B.n; i++) v[i] = B.U[i].d;
    CKR(cudaMemcpyAsync(B.dU, v.data(), sizeof(UniDev) * B.n, cudaMemcpyHostToDevice, B.st));
    B.h2d += sizeof(UniDev) * B.n;
    CKR(cudaStreamSynchronize(B.st));
    return UG_OK;
}

// ---------------------------------------------------------- round launch

static int launch_round(Batch& B, bool timed) {
    B.synced = false;
    auto tb = [&](int k) {
        if (timed) cudaEventRecord(B.ev[2 * k], B.st);
    };
    auto te = [&](int k) {
        if (timed) {
            cudaEventRecord(B.ev[2 * k + 1], B.st);
            cudaEventSynchronize(B.ev[2 * k + 1]);
            float ms = 0;
            cudaEventElapsedTime(&ms, B.ev[2 * k], B.ev[2 * k + 1]);
            B.kms[k] += ms;
            B.klaunch[k]++;
        }
    };
    tb(K_PLAN);
    k_plan<<<1, 256, 0, B.st>>>(B.dU, B.dCtl, B.dInfo);
    te(K_PLAN);
    if (B.opts.precision == UG_PREC_MIXED && B.any_mixed) {
        tb(K_MIXED);
        launch_prefilter_mixed(B.dU, B.dCtl, B.dInfo, B.nsm, B.any_group, B.any_euclid, B.st);
        te(K_MIXED);
        tb(K_CONFIRM);
        k_gray_compact<<<B.n, 256, 0, B.st>>>(B.dU, B.dCtl, B.dInfo, 0);
        // the retest: few candidates per round, a block of warps per candidate
        launch_confirm64w(0, B.nsm, B.dU, B.dCtl, B.dInfo, B.st);
        te(K_CONFIRM);
    } else {
        // the FP64 form: every candidate of the round, one warp per candidate
        // (coefficients in shared memory, lanes over timesteps in endpoint-first order)
        tb(K_PRE);
        k_gray_compact<<<B.n, 256, 0, B.st>>>(B.dU, B.dCtl, B.dInfo, 1);
        launch_confirm64w(1, B.nsm, B.dU, B.dCtl, B.dInfo, B.st);
        te(K_PRE);
    }
    tb(K_COMPACT);
    k_compact<<<B.n, 256, 0, B.st>>>(B.dU, B.dCtl, B.dInfo);
    te(K_COMPACT);
    tb(K_SGEN);
    {
        const int wb = (int)(B.any_knot ? kSurvSmemPerWarp : kSurvSmemAxis);
        k_surv_gen<<<B.nsm * B.res_sgen, 32 * kSurvWarps, kSurvWarps * wb, B.st>>>(B.dU, B.dCtl, B.dInfo, wb);
    }
    te(K_SGEN);
    tb(K_SGEMM);
    k_surv_gemm<<<B.nsm * 4, 128, kGemmSmem, B.st>>>(B.dU, B.dCtl, B.dInfo);
    te(K_SGEMM);
    tb(K_SHASH);
    k_surv_hash<<<B.nsm * B.res_shash, 256, 0, B.st>>>(B.dU, B.dCtl, B.dInfo);
    te(K_SHASH);
    tb(K_CONFL);
    k_conflicts<<<B.nsm * B.res_confl, 128, 0, B.st>>>(B.dU, B.dCtl, B.dInfo);
    te(K_CONFL);
    tb(K_GREEDY);
    k_greedy<<<B.n, 32, 2 * kSmaxCap * sizeof(int32_t), B.st>>>(B.dU, B.dCtl, B.dInfo);
    te(K_GREEDY);
    tb(K_COMMIT);
    k_commit<<<B.nsm * 8, 256, 0, B.st>>>(B.dU, B.dCtl, B.dInfo);
    te(K_COMMIT);
    CKR(cudaGetLastError());
    return UG_OK;
}

static int build_graph(Batch& B, int rounds) {
    if (B.gexec) {
        cudaGraphExecDestroy(B.gexec);
        B.gexec = nullptr;
    }
    cudaGraph_t g;
    CKR(cudaStreamBeginCapture(B.st, cudaStreamCaptureModeThreadLocal));
    for (int r = 0; r < rounds; r++) {
        int rc = launch_round(B, false);
        if (rc) {
            cudaStreamEndCapture(B.st, &g);
            return rc;
        }
    }
    CKR(cudaStreamEndCapture(B.st, &g));
    CKR(cudaGraphInstantiate(&B.gexec, g, 0));
    CKR(cudaGraphDestroy(g));
    B.graph_rounds = rounds;
    return UG_OK;
}

// Host snapshot of the control blocks.  Work that may change them clears
// B.synced; reads that find it set use the snapshot without a copy.
static int pull_ctl(Batch& B) {
    if (B.synced) return UG_OK;
    CKR(cudaMemcpyAsync(B.hCtl.data(), B.dCtl, sizeof(UniCtl) * B.n, cudaMemcpyDeviceToHost, B.st));
    B.d2h += sizeof(UniCtl) * B.n;
    CKR(cudaStreamSynchronize(B.st));
#ifdef UG_CHECKED
    unsigned long long rec[4] = {0, 0, 0, 0};
    CKR(cudaMemcpyFromSymbol(rec, ug_check_record, sizeof rec));
    if (rec[3])
        return fail(UG_ECAP, "index guard: source line %llu index %lld bound %lld", rec[0], (long long)rec[1],
                    (long long)rec[2]);
#endif
    B.synced = true;
    return UG_OK;
}

// Grow slot / hash capacity ahead of the next `rounds` rounds.
static int ensure_capacity(Batch& B, int rounds) {
    bool changed = false;
    for (int i = 0; i < B.n; i++) {
        UniHost& h = B.U[i];
        UniCtl& k = B.hCtl[i];
        if (k.state == ST_ERROR) return fail(UG_ECAP, "universe %d: device error %d", i, k.err_code);
        if (k.state == ST_DONE) continue;
        const int64_t need = k.n_slots + std::max<int64_t>(h.d.S_max, (int64_t)rounds * h.d.S_max / 4);
        if (need > h.d.slot_cap || k.state == ST_GROW) {
            int64_t ncap = std::max<int64_t>(h.d.slot_cap * 2, need);
            const int T = h.cfg.T;
            Pt64* op = h.d.pts;
            Pt32* of = h.d.ptf;
            int64_t* oi = h.d.acc_idx;
            const int64_t n = k.n_slots;
            int rc = alloc_points(h, ncap);
            if (rc) return rc;
            CKR(cudaMemcpyAsync(h.d.pts, op, (size_t)n * T * sizeof(Pt64), cudaMemcpyDeviceToDevice, B.st));
            CKR(cudaMemcpyAsync(h.d.ptf, of, (size_t)n * T * sizeof(Pt32), cudaMemcpyDeviceToDevice, B.st));
            CKR(cudaMemcpyAsync(h.d.acc_idx, oi, (size_t)n * sizeof(int64_t), cudaMemcpyDeviceToDevice, B.st));
            CKR(cudaStreamSynchronize(B.st));
            cudaFree(op);
            cudaFree(of);
            cudaFree(oi);
            if (k.state == ST_GROW) {
                k.state = ST_ACTIVE;
                CKR(cudaMemcpyAsync(&B.dCtl[i].state, &k.state, sizeof(int32_t), cudaMemcpyHostToDevice, B.st));
            }
            changed = true;
        }
        if (h.d.grid_kind == GRID_HASH) {
            const int64_t need_keys = k.hash_used + (int64_t)rounds * h.d.S_max * h.cfg.T;
            if (need_keys * 2 > h.hcap) {
                ulonglong2* os = h.d.hslot;
                int rc = alloc_hash(h, pow2_at_least(need_keys * 4));
                if (rc) return rc;
                cudaFree(os);
                int64_t zero = 0;
                k.hash_used = 0;
                CKR(cudaMemcpyAsync(&B.dCtl[i].hash_used, &zero, sizeof zero, cudaMemcpyHostToDevice, B.st));
                changed = true;
                int rc2 = push_unidev(B);
                if (rc2) return rc2;
                if (k.n_slots > 0) {
                    B.synced = false;
                    k_rehash<<<B.nsm * 4, 256, 0, B.st>>>(B.dU, B.dCtl, i, k.n_slots);
                }
                CKR(cudaGetLastError());
                CKR(cudaStreamSynchronize(B.st));
            }
        }
    }
    if (changed) return push_unidev(B);
    return UG_OK;
}

static bool all_done(const Batch& B) {
    for (const UniCtl& k : B.hCtl)
        if (k.state != ST_DONE) return false;
    return true;
}

}  // namespace ug

// Internal accessor for ug_noalloc.cu: what a parameter dump of universe u
// needs, without allocating anything.
namespace ug {
int batch_params_view(void* h, int u, const UniDev** dU, int64_t* n, int* dim, int* nw, int* dev,
                      cudaStream_t* st) {
    Batch* B = (Batch*)h;
    if (!B || u < 0 || u >= B->n) return fail(UG_EINVAL, "bad arguments");
    int rc = pull_ctl(*B);
    if (rc) return rc;
    *dU = B->dU;
    *n = B->hCtl[u].n_slots;
    *dim = B->U[u].d.dim;
    *nw = B->U[u].d.nw;
    *dev = B->dev;
    *st = B->st;
    return UG_OK;
}
int set_error(int code, const char* msg) { return fail(code, "%s", msg); }
}  // namespace ug

using namespace ug;

extern "C" {

int ug_version(void) { return 1; }

int ug_device_info(int32_t device, char* name, size_t len, int32_t* sms) {
    int dev = device;
    if (dev < 0 && cudaGetDevice(&dev) != cudaSuccess) return fail(UG_ECUDA, "no current device");
    cudaDeviceProp prop;
    const cudaError_t e = cudaGetDeviceProperties(&prop, dev);
    if (e != cudaSuccess) return fail(UG_ECUDA, "cudaGetDeviceProperties(%d): %s", dev, cudaGetErrorString(e));
    if (name && len) {
        snprintf(name, len, "%s sm_%d%d", prop.name, prop.major, prop.minor);
    }
    if (sms) *sms = prop.multiProcessorCount;
    return UG_OK;
}

int ug_selftest_bounded_wait(int64_t limit_ns, int32_t* status) {
    if (!status || limit_ns < 0 || limit_ns > 10000000000ll) return fail(UG_EINVAL, "bad arguments");
    const int rc = wait_selftest(limit_ns, status);
    return rc ? fail(rc, "bounded-wait self-test: %s", cudaGetErrorString(cudaGetLastError())) : UG_OK;
}

int ug_struct_sizes(int64_t* sizes, int32_t n) {
    const int64_t v[7] = {(int64_t)sizeof(ug_universe_cfg), (int64_t)sizeof(ug_run_opts), (int64_t)sizeof(ug_stats),
                          (int64_t)sizeof(ug_kernel_times), (int64_t)sizeof(ug_hit), (int64_t)sizeof(ug_frames_cfg),
                          (int64_t)sizeof(ug_frames_out)};
    for (int i = 0; sizes && i < n && i < 7; i++) sizes[i] = v[i];
    return 7;
}

int ug_last_error(char* buf, size_t len) {
    if (buf && len) {
        strncpy(buf, g_err.c_str(), len - 1);
        buf[len - 1] = 0;
    }
    return (int)g_err.size();
}

int ug_batch_create(const ug_universe_cfg* cfgs, int32_t n, const ug_run_opts* opts, void** out) {
    if (!cfgs || !out || n < 1 || n > kMaxUni) return fail(UG_EINVAL, "bad batch arguments (n=%d)", n);
    for (int i = 0; i < n; i++) {
        int rc = validate(cfgs[i]);
        if (rc) return rc;
    }
    Batch* B = new Batch();
    if (opts) B->opts = *opts;
    if (B->opts.rounds_per_sync <= 0) B->opts.rounds_per_sync = 8;
    if (B->opts.device >= 0) {
        cudaError_t e = cudaSetDevice(B->opts.device);
        if (e != cudaSuccess) {
            delete B;
            return fail(UG_ECUDA, "cudaSetDevice(%d): %s", B->opts.device, cudaGetErrorString(e));
        }
    }
    cudaGetDevice(&B->dev);
    cudaDeviceGetAttribute(&B->nsm, cudaDevAttrMultiProcessorCount, B->dev);
    int rc = UG_OK;
    auto bail = [&](int code) {
        ug_batch_destroy(B);
        return code;
    };
    if (B->opts.stream) {
        B->st = (cudaStream_t)(uintptr_t)B->opts.stream;
    } else {
        if (cudaStreamCreateWithFlags(&B->st, cudaStreamNonBlocking) != cudaSuccess)
            return bail(fail(UG_ECUDA, "stream create failed"));
        B->own_stream = true;
    }
    B->n = n;
    B->U.resize(n);
    size_t freeb = 0, totalb = 0;
    cudaMemGetInfo(&freeb, &totalb);
    const int64_t dense_budget = (int64_t)(freeb * 0.35);
    int64_t dense_used = 0;
    for (int i = 0; i < n; i++) {
        B->U[i].cfg = cfgs[i];
        B->max_T = std::max(B->max_T, cfgs[i].T);
        if ((rc = setup_universe(*B, B->U[i], dense_budget, &dense_used))) return bail(rc);
        if (B->opts.precision == UG_PREC_MIXED) {
            if ((rc = mixed_setup(B->U[i].cfg, B->U[i].d, B->U[i].mt))) return bail(rc);
            B->any_mixed = true;
        }
        if (cfgs[i].group_mode != UG_GROUP_NONE) B->any_group = true;
        if (cfgs[i].euclid) B->any_euclid = true;
        if (cfgs[i].rng == UG_RNG_KNOT) B->any_knot = true;
    }
    if (cudaMalloc(&B->dU, sizeof(UniDev) * n) != cudaSuccess ||
        cudaMalloc(&B->dCtl, sizeof(UniCtl) * n) != cudaSuccess ||
        cudaMalloc(&B->dInfo, sizeof(RoundInfo)) != cudaSuccess)
        return bail(fail(UG_ENOMEM, "control block allocation failed"));
    B->hCtl.resize(n);
    for (int i = 0; i < n; i++) init_ctl(cfgs[i], B->U[i].d, B->hCtl[i]);
    RoundInfo ri;
    memset(&ri, 0, sizeof ri);
    ri.n_uni = n;
    if (cudaMemcpy(B->dCtl, B->hCtl.data(), sizeof(UniCtl) * n, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(B->dInfo, &ri, sizeof ri, cudaMemcpyHostToDevice) != cudaSuccess)
        return bail(fail(UG_ECUDA, "control block upload failed"));
    if ((rc = push_unidev(*B))) return bail(rc);
    if (cudaFuncSetAttribute(k_greedy, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(2 * kSmaxCap * sizeof(int32_t))) != cudaSuccess)
        return bail(fail(UG_ECUDA, "smem attribute failed"));
    if (cudaFuncSetAttribute(k_surv_gen, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(kSurvWarps * kSurvSmemPerWarp)) != cudaSuccess ||
        cudaFuncSetAttribute(k_restore_gen, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(kSurvWarps * kSurvSmemPerWarp)) != cudaSuccess)
        return bail(fail(UG_ECUDA, "smem attribute failed"));
    if (B->any_mixed && (rc = mixed_init_kernels())) return bail(rc);
    B->kernels_per_round = B->any_mixed ? 11 : 10;
    // the warp FP64 test serves both forms (all candidates, or the undecided ones)
    if (confirm64w_set_smem() != cudaSuccess)
        return bail(fail(UG_ECUDA, "smem attribute failed"));
    // one wave per SM, measured on c3 against 8 / 8 / 16 CTAs per SM: k_surv_gen 27.7 ->
    // 24.5 ms, k_surv_hash 33.5 -> 32.0 ms, k_conflicts 85.5 -> 80.2 ms per job.  k_commit
    // and k_confirm64w keep 8 and 4 per SM (more than resident): one wave measured slower
    // for them (56.6 -> 60.0 and 38.2 -> 40.6 ms).
    B->res_sgen = resident_ctas(k_surv_gen, 32 * kSurvWarps,
                                kSurvWarps * (B->any_knot ? kSurvSmemPerWarp : kSurvSmemAxis), 8);
    B->res_shash = resident_ctas(k_surv_hash, 256, 0, 8);
    B->res_confl = resident_ctas(k_conflicts, 128, 0, 16);
    for (int k = 0; k < 2 * K_NK; k++) cudaEventCreate(&B->ev[k]);
    *out = B;
    return UG_OK;
}

int ug_batch_run(void* h, int64_t max_rounds) {
    Batch* B = (Batch*)h;
    if (!B) return fail(UG_EINVAL, "null handle");
    int rc = pull_ctl(*B);
    if (rc) return rc;
    int64_t done_rounds = 0;
    const int R = B->opts.rounds_per_sync;
    int stalls = 0;
    while (!all_done(*B)) {
        int64_t progress_before = 0;
        for (const UniCtl& k : B->hCtl) progress_before += k.next_cand + k.n_slots;
        if (max_rounds > 0 && done_rounds >= max_rounds) return UG_OK;
        if ((rc = ensure_capacity(*B, R))) return rc;
        if (B->opts.use_graph && !B->opts.kernel_timing) {
            if (!B->gexec && (rc = build_graph(*B, R))) return rc;
            B->synced = false;
            CKR(cudaGraphLaunch(B->gexec, B->st));
        } else {
            for (int r = 0; r < R; r++)
                if ((rc = launch_round(*B, B->opts.kernel_timing != 0))) return rc;
        }
        B->launches += (int64_t)R * B->kernels_per_round;
        done_rounds += R;
        if ((rc = pull_ctl(*B))) return rc;
        int64_t progress_after = 0;
        for (const UniCtl& k : B->hCtl) progress_after += k.next_cand + k.n_slots;
        stalls = progress_after == progress_before ? stalls + 1 : 0;
        if (stalls > 64) return fail(UG_ETIMEDOUT, "no universe made progress in %d rounds", 64 * R);
    }
    return UG_OK;
}

int ug_batch_reset(void* h, const uint64_t* seeds) {
    Batch* B = (Batch*)h;
    if (!B) return fail(UG_EINVAL, "null handle");
    CKR(cudaStreamSynchronize(B->st));
    for (int i = 0; i < B->n; i++) {
        UniHost& u = B->U[i];
        if (seeds) {
            u.cfg.seed = seeds[i];
            u.d.seed = seeds[i];
        }
        if (u.d.grid_kind == GRID_DENSE) {
            int64_t cpt = 1;
            for (int ax = 0; ax < u.d.dim; ax++) cpt *= u.d.gw;
            CKR(cudaMemsetAsync(u.d.heads, 0xff, (size_t)u.d.T * cpt * sizeof(int32_t), B->st));
        } else {
            CKR(cudaMemsetAsync(u.d.hslot, 0xff, (size_t)u.hcap * sizeof(ulonglong2), B->st));
        }
        CKR(cudaMemsetAsync(u.d.occ, 0, (size_t)u.occ_words * sizeof(uint32_t), B->st));
        CKR(cudaMemsetAsync(u.d.occ1, 0, (size_t)u.occ1_words * sizeof(uint32_t), B->st));
        const int32_t ep = B->hCtl[i].epoch;
        init_ctl(u.cfg, u.d, B->hCtl[i]);
        B->hCtl[i].epoch = ep;  // round-table entries of earlier epochs stay stale
    }
    B->synced = false;
    CKR(cudaMemcpyAsync(B->dCtl, B->hCtl.data(), sizeof(UniCtl) * B->n, cudaMemcpyHostToDevice, B->st));
    B->h2d += sizeof(UniCtl) * B->n;
    return push_unidev(*B);
}

int ug_batch_done(void* h) {
    Batch* B = (Batch*)h;
    if (!B) return -UG_EINVAL;
    if (pull_ctl(*B)) return -UG_ECUDA;
    return all_done(*B) ? 1 : 0;
}

int ug_batch_stats(void* h, int32_t u, ug_stats* out) {
    Batch* B = (Batch*)h;
    if (!B || u < 0 || u >= B->n || !out) return fail(UG_EINVAL, "bad arguments");
    int rc = pull_ctl(*B);
    if (rc) return rc;
    const UniCtl& k = B->hCtl[u];
    out->n = k.n_slots;
    out->n_unique = k.n_unique;
    out->n_sub = k.n_sub;
    out->attempts = k.attempts;
    out->phase1_end = k.phase == 2 ? k.phase1_end : k.attempts;
    out->rounds = k.rounds;
    out->gray = k.gray_total;
    out->evals = k.evals;
    out->evals_fp64 = k.evals_fp64;
    out->state = k.state;
    out->grid_kind = B->U[u].d.grid_kind;
    out->filled = k.filled + k.round_new;
    out->visits = k.visits;
    return UG_OK;
}

int ug_batch_accepted(void* h, int32_t u, int64_t* idx, int32_t* gid, int64_t cap, int64_t* n) {
    Batch* B = (Batch*)h;
    if (!B || u < 0 || u >= B->n) return fail(UG_EINVAL, "bad arguments");
    int rc = pull_ctl(*B);
    if (rc) return rc;
    const int64_t N = B->hCtl[u].n_slots;
    if (n) *n = N;
    if (cap <= 0) return UG_OK;
    if (cap < N) return fail(UG_ECAP, "accepted buffer too small (%lld < %lld)", (long long)cap, (long long)N);
    const UniDev& d = B->U[u].d;
    if (idx && N) CKR(cudaMemcpy(idx, d.acc_idx, N * sizeof(int64_t), cudaMemcpyDeviceToHost));
    if (idx) B->d2h += N * sizeof(int64_t);
    if (gid && N) {
        std::vector<Pt64> tmp(N);
        CKR(cudaMemcpy2D(tmp.data(), sizeof(Pt64), d.pts, sizeof(Pt64) * d.T, sizeof(Pt64), N,
                         cudaMemcpyDeviceToHost));
        B->d2h += N * sizeof(Pt64);
        for (int64_t i = 0; i < N; i++) gid[i] = tmp[i].gid;
    }
    return UG_OK;
}

int ug_batch_accepted_all(void* h, int64_t* idx, int32_t* gid, int64_t cap, int64_t* counts) {
    Batch* B = (Batch*)h;
    if (!B || !counts) return fail(UG_EINVAL, "bad arguments");
    int rc = pull_ctl(*B);
    if (rc) return rc;
    std::vector<int64_t> off(B->n + 1, 0);
    for (int u = 0; u < B->n; u++) {
        counts[u] = B->hCtl[u].n_slots;
        off[u + 1] = off[u] + counts[u];
    }
    const int64_t total = off[B->n];
    if (cap <= 0 || total == 0) return UG_OK;
    if (cap < total) return fail(UG_ECAP, "accepted buffer too small (%lld < %lld)", (long long)cap, (long long)total);
    if (total > B->gather_cap) {
        cudaFree(B->d_gather_idx);
        cudaFree(B->d_gather_gid);
        B->d_gather_idx = nullptr;
        B->d_gather_gid = nullptr;
        const int64_t c = pow2_at_least(total);
        CKR(cudaMalloc(&B->d_gather_idx, (size_t)c * sizeof(int64_t)));
        CKR(cudaMalloc(&B->d_gather_gid, (size_t)c * sizeof(int32_t)));
        B->gather_cap = c;
    }
    if (!B->d_gather_off) CKR(cudaMalloc(&B->d_gather_off, (size_t)(kMaxUni + 1) * sizeof(int64_t)));
    CKR(cudaMemcpyAsync(B->d_gather_off, off.data(), off.size() * sizeof(int64_t), cudaMemcpyHostToDevice, B->st));
    B->h2d += off.size() * sizeof(int64_t);
    k_gather_accepted<<<B->n, 256, 0, B->st>>>(B->dU, B->d_gather_off, B->d_gather_idx, B->d_gather_gid);
    CKR(cudaGetLastError());
    B->launches++;
    if (idx) {
        CKR(cudaMemcpyAsync(idx, B->d_gather_idx, (size_t)total * sizeof(int64_t), cudaMemcpyDeviceToHost, B->st));
        B->d2h += total * sizeof(int64_t);
    }
    if (gid) {
        CKR(cudaMemcpyAsync(gid, B->d_gather_gid, (size_t)total * sizeof(int32_t), cudaMemcpyDeviceToHost, B->st));
        B->d2h += total * sizeof(int32_t);
    }
    CKR(cudaStreamSynchronize(B->st));
    return UG_OK;
}

int ug_batch_positions(void* h, int32_t u, double* pos, int64_t cap_paths) {
    Batch* B = (Batch*)h;
    if (!B || u < 0 || u >= B->n || !pos) return fail(UG_EINVAL, "bad arguments");
    int rc = pull_ctl(*B);
    if (rc) return rc;
    const int64_t N = B->hCtl[u].n_slots;
    if (cap_paths < N) return fail(UG_ECAP, "positions buffer too small");
    const UniDev& d = B->U[u].d;
    std::vector<Pt64> tmp((size_t)N * d.T);
    if (N) CKR(cudaMemcpy(tmp.data(), d.pts, tmp.size() * sizeof(Pt64), cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < N; i++)
        for (int ax = 0; ax < d.dim; ax++)
            for (int t = 0; t < d.T; t++) pos[(i * d.dim + ax) * d.T + t] = tmp[(size_t)i * d.T + t].c[ax];
    return UG_OK;
}

int ug_batch_params(void* h, int32_t u, double* a2, double* a, int32_t* b, double* f, int64_t cap_paths) {
    Batch* B = (Batch*)h;
    if (!B || u < 0 || u >= B->n) return fail(UG_EINVAL, "bad arguments");
    int rc = pull_ctl(*B);
    if (rc) return rc;
    const int64_t N = B->hCtl[u].n_slots;
    if (cap_paths < N) return fail(UG_ECAP, "params buffer too small");
    if (N == 0) return UG_OK;
    const UniDev& d = B->U[u].d;
    const int nw = d.nw, D = d.dim;
    double *da2, *da, *df;
    int32_t* db;
    CKR(cudaMalloc(&da2, (size_t)N * D * 8));
    CKR(cudaMalloc(&da, (size_t)N * D * nw * 8));
    CKR(cudaMalloc(&df, (size_t)N * D * nw * 8));
    CKR(cudaMalloc(&db, (size_t)N * D * nw * 4));
    launch_params(B->dU, u, N, da2, da, db, df, B->st);
    cudaError_t e = cudaStreamSynchronize(B->st);
    if (e == cudaSuccess && a2) e = cudaMemcpy(a2, da2, (size_t)N * D * 8, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && a) e = cudaMemcpy(a, da, (size_t)N * D * nw * 8, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && f) e = cudaMemcpy(f, df, (size_t)N * D * nw * 8, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && b) e = cudaMemcpy(b, db, (size_t)N * D * nw * 4, cudaMemcpyDeviceToHost);
    cudaFree(da2);
    cudaFree(da);
    cudaFree(df);
    cudaFree(db);
    if (e != cudaSuccess) return fail(UG_ECUDA, "params: %s", cudaGetErrorString(e));
    return UG_OK;
}

int ug_batch_frames(void* h, int32_t u, const ug_frames_cfg* cfg, ug_frames_out* out) {
    Batch* B = (Batch*)h;
    if (!B || u < 0 || u >= B->n || !cfg || !out) return fail(UG_EINVAL, "bad arguments");
    if (B->U[u].cfg.dim != 2) return fail(UG_ENOTSUP, "frames are baked for 2+1 universes");
    int rc = pull_ctl(*B);
    if (rc) return rc;
    const int64_t N = B->hCtl[u].n_slots;
    if (N < 1) return fail(UG_EINVAL, "frames: the universe has no accepted paths");
    if (N > INT32_MAX / 2) return fail(UG_ECAP, "frames: too many paths");
    const int nw = B->U[u].d.nw;
    double *da2 = nullptr, *da = nullptr, *df = nullptr;
    int32_t* db = nullptr;
    auto release = [&]() {
        cudaFree(da2);
        cudaFree(da);
        cudaFree(df);
        cudaFree(db);
    };
    if (cudaMalloc(&da2, (size_t)N * 2 * 8) != cudaSuccess || cudaMalloc(&da, (size_t)N * 2 * nw * 8) != cudaSuccess ||
        cudaMalloc(&df, (size_t)N * 2 * nw * 8) != cudaSuccess || cudaMalloc(&db, (size_t)N * 2 * nw * 4) != cudaSuccess) {
        release();
        return fail(UG_ENOMEM, "frames: device allocation failed");
    }
    launch_params(B->dU, u, N, da2, da, db, df, B->st);
    int bMax = 2;
    if (cudaStreamSynchronize(B->st) != cudaSuccess || (rc = max_b_device(db, N * 2 * nw, &bMax, B->st))) {
        release();
        return rc ? rc : fail(UG_ECUDA, "frames: parameter kernel failed");
    }
    rc = frames_from_params(cfg, (int)N, nw, bMax, da2, da, db, df, out, B->st);
    release();
    return rc;
}

int ug_batch_probe(void* h, int32_t u, uint64_t seed, int64_t n, int32_t bins, int64_t* proposed,
                   int64_t* accepted) {
    Batch* B = (Batch*)h;
    if (!B || u < 0 || u >= B->n || n < 0 || bins < 1 || bins > 4096 || !proposed || !accepted)
        return fail(UG_EINVAL, "bad arguments");
    int rc = pull_ctl(*B);
    if (rc) return rc;
    unsigned long long* dh = nullptr;
    CKR(cudaMalloc(&dh, sizeof(unsigned long long) * 2 * bins));
    cudaError_t e = cudaMemsetAsync(dh, 0, sizeof(unsigned long long) * 2 * bins, B->st);
    if (e == cudaSuccess && n > 0) {
        const int blocks = (int)std::min<int64_t>((n + kTile - 1) / kTile, (int64_t)B->nsm * 16);
        k_probe<<<blocks, kTile, sizeof(unsigned long long) * 2 * bins, B->st>>>(
            B->dU, u, B->hCtl[u].n_slots, seed, n, bins, dh, dh + bins);
        e = cudaGetLastError();
    }
    std::vector<unsigned long long> hh(2 * bins);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(hh.data(), dh, sizeof(unsigned long long) * 2 * bins, cudaMemcpyDeviceToHost, B->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(B->st);
    cudaFree(dh);
    if (e != cudaSuccess) return fail(UG_ECUDA, "probe: %s", cudaGetErrorString(e));
    for (int i = 0; i < bins; i++) {
        proposed[i] = (int64_t)hh[i];
        accepted[i] = (int64_t)hh[bins + i];
    }
    return UG_OK;
}

// ---------------------------------------------------------- checkpoints

namespace {
// Saved control block of one universe: what it was built from, then the block.
struct CkHeader {
    char magic[4];  // "UGCK"
    int32_t version;
    int32_t ctl_bytes;
    int32_t pad;
    ug_universe_cfg cfg;
};
constexpr int32_t kCkVersion = 1;

bool same_model(const ug_universe_cfg& a, const ug_universe_cfg& b) {
    return a.dim == b.dim && a.T == b.T && a.terms == b.terms && a.rng == b.rng && a.zgrid == b.zgrid &&
           a.excl == b.excl && a.cross1d == b.cross1d && a.pin_sin1 == b.pin_sin1 && a.group_mode == b.group_mode &&
           a.seed == b.seed && a.euclid == b.euclid;
}
}  // namespace

int64_t ug_state_bytes(void) { return (int64_t)(sizeof(CkHeader) + sizeof(UniCtl)); }

int ug_batch_save_state(void* h, int32_t u, void* buf) {
    Batch* B = (Batch*)h;
    if (!B || u < 0 || u >= B->n || !buf) return fail(UG_EINVAL, "bad arguments");
    int rc = pull_ctl(*B);
    if (rc) return rc;
    CkHeader hd{};
    memcpy(hd.magic, "UGCK", 4);
    hd.version = kCkVersion;
    hd.ctl_bytes = (int32_t)sizeof(UniCtl);
    hd.cfg = B->U[u].cfg;
    memcpy(buf, &hd, sizeof hd);
    memcpy((char*)buf + sizeof hd, &B->hCtl[u], sizeof(UniCtl));
    return UG_OK;
}

// Rebuilds universe u from its admissions (candidate indices in admission order
// and their groups) and a saved control block: the trajectories are regenerated
// from the candidate stream and appended to a cleared grid in admission order,
// S_max paths per step, by the survivor product and commit kernels.
int ug_batch_restore(void* h, int32_t u, int64_t n, const int64_t* idx, const int32_t* gid, const void* buf) {
    Batch* B = (Batch*)h;
    if (!B || u < 0 || u >= B->n || !buf || n < 0 || (n > 0 && (!idx || !gid)))
        return fail(UG_EINVAL, "bad arguments");
    CkHeader hd;
    memcpy(&hd, buf, sizeof hd);
    if (memcmp(hd.magic, "UGCK", 4) || hd.version != kCkVersion || hd.ctl_bytes != (int32_t)sizeof(UniCtl))
        return fail(UG_EINVAL, "restore: not a state of this library version");
    UniHost& U = B->U[u];
    if (!same_model(hd.cfg, U.cfg)) return fail(UG_EINVAL, "restore: the state belongs to another universe model");
    UniCtl saved;
    memcpy(&saved, (const char*)buf + sizeof hd, sizeof saved);
    if (saved.n_slots != n) return fail(UG_EINVAL, "restore: %lld admissions given, the state has %lld",
                                        (long long)n, (long long)saved.n_slots);
    if (saved.state == ST_ERROR) return fail(UG_EINVAL, "restore: the saved universe had failed");
    int rc = pull_ctl(*B);
    if (rc) return rc;
    UniDev& d = U.d;
    const int T = U.cfg.T;
    // clear the universe's grid, bitmaps and round table
    if (d.grid_kind == GRID_DENSE) {
        int64_t cpt = 1;
        for (int ax = 0; ax < d.dim; ax++) cpt *= d.gw;
        CKR(cudaMemsetAsync(d.heads, 0xff, (size_t)T * cpt * sizeof(int32_t), B->st));
    } else {
        const int64_t need = std::max<int64_t>(1 << 16, pow2_at_least((n * T + (int64_t)d.S_max * T) * 4));
        if (need > U.hcap) {
            CKR(cudaStreamSynchronize(B->st));
            cudaFree(d.hslot);
            if ((rc = alloc_hash(U, need))) return rc;
        } else {
            CKR(cudaMemsetAsync(d.hslot, 0xff, (size_t)U.hcap * sizeof(ulonglong2), B->st));
        }
    }
    CKR(cudaMemsetAsync(d.occ, 0, (size_t)U.occ_words * sizeof(uint32_t), B->st));
    CKR(cudaMemsetAsync(d.occ1, 0, (size_t)U.occ1_words * sizeof(uint32_t), B->st));
    CKR(cudaMemsetAsync(d.rhead, 0xff, (size_t)T * d.rblocks * sizeof(uint64_t), B->st));
    // room for the admissions and the next rounds
    if (n + (int64_t)d.S_max * 2 > d.slot_cap) {
        CKR(cudaStreamSynchronize(B->st));
        cudaFree(d.pts);
        cudaFree(d.ptf);
        cudaFree(d.acc_idx);
        if ((rc = alloc_points(U, n + (int64_t)d.S_max * 2))) return rc;
    }
    if ((rc = push_unidev(*B))) return rc;
    // rebuild control block: k_commit reads these and accumulates hash keys and cells
    UniCtl k = B->hCtl[u];
    B->synced = false;
    const int32_t epoch = k.epoch;
    init_ctl(U.cfg, d, k);
    k.epoch = epoch;
    k.state = ST_ACTIVE;
    std::vector<int32_t> iota(d.S_max), zero(d.S_max + 1, 0);
    for (int i = 0; i < d.S_max; i++) iota[i] = i;
    int64_t* dIdx = nullptr;
    CKR(cudaMalloc(&dIdx, (size_t)d.S_max * sizeof(int64_t)));
    RoundInfo* ri = new RoundInfo();
    int64_t done = 0;
    while (done < n && rc == UG_OK) {
        const int m = (int)std::min<int64_t>(d.S_max, n - done);
        k.S = k.S_raw = k.trunc = k.stop_at = m;
        k.n_slots_prev = done;
        k.n_slots = done;
        k.round_base = 0;
        memset(ri, 0, sizeof(RoundInfo));
        ri->n_uni = B->n;
        const int sev = ((m * d.dim + 31) >> 5) * ((T + 31) >> 5);
        for (int v = 0; v <= B->n; v++) {
            const bool past = v > u;
            ri->surv_off[v] = past ? m : 0;
            ri->sev_off[v] = past ? sev : 0;
            ri->sev_off_o[v] = past ? sev : 0;
            ri->spt_off[v] = past ? m * T : 0;
            if (v < B->n) ri->tile_uni[v] = v;  // tile order = universe order here
        }
        ri->total_surv = m;
        ri->total_sev = sev;
        ri->total_spt = m * T;
        cudaError_t e = cudaMemcpyAsync(B->dInfo, ri, sizeof(RoundInfo), cudaMemcpyHostToDevice, B->st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&B->dCtl[u], &k, sizeof(UniCtl), cudaMemcpyHostToDevice, B->st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(d.acc_rank, iota.data(), (size_t)m * 4, cudaMemcpyHostToDevice, B->st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(d.sgid, gid + done, (size_t)m * 4, cudaMemcpyHostToDevice, B->st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(d.surv_off, zero.data(), (size_t)(m + 1) * 4, cudaMemcpyHostToDevice, B->st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(dIdx, idx + done, (size_t)m * 8, cudaMemcpyHostToDevice, B->st);
        if (e == cudaSuccess) e = cudaMemsetAsync(d.spos, 0, (size_t)m * T * sizeof(Pt64), B->st);  // unused axes
        if (e == cudaSuccess) {
            k_restore_gen<<<B->nsm * 4, 32 * kSurvWarps, kSurvWarps * kSurvSmemPerWarp, B->st>>>(B->dU, u, dIdx, m);
            k_surv_gemm<<<B->nsm * 4, 128, kGemmSmem, B->st>>>(B->dU, B->dCtl, B->dInfo);
            k_commit<<<B->nsm * 8, 256, 0, B->st>>>(B->dU, B->dCtl, B->dInfo);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(d.acc_idx + done, dIdx, (size_t)m * 8, cudaMemcpyDeviceToDevice, B->st);
        // carry the device-accumulated counters into the next step's block
        if (e == cudaSuccess) e = cudaMemcpyAsync(&k, &B->dCtl[u], sizeof(UniCtl), cudaMemcpyDeviceToHost, B->st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(B->st);
        if (e != cudaSuccess) rc = fail(UG_ECUDA, "restore: %s", cudaGetErrorString(e));
        else if (k.state == ST_ERROR) rc = fail(UG_ECAP, "restore: device error %d", k.err_code);
        done += m;
    }
    delete ri;
    cudaFree(dIdx);
    if (rc) return rc;
    const int64_t filled = k.filled + k.round_new;
    if (filled != saved.filled + saved.round_new)
        return fail(UG_EINVAL, "restore: rebuilt grid holds %lld cells, the state %lld (admissions do not match)",
                    (long long)filled, (long long)(saved.filled + saved.round_new));
    // the saved block, with this batch's hash usage and round-table epoch
    saved.hash_used = k.hash_used;
    saved.epoch = epoch;
    B->hCtl[u] = saved;
    CKR(cudaMemcpyAsync(&B->dCtl[u], &saved, sizeof(UniCtl), cudaMemcpyHostToDevice, B->st));
    CKR(cudaStreamSynchronize(B->st));
    return UG_OK;
}

int ug_batch_kernel_times(void* h, ug_kernel_times* out) {
    Batch* B = (Batch*)h;
    if (!B || !out) return fail(UG_EINVAL, "bad arguments");
    memset(out, 0, sizeof *out);
    for (int k = 0; k < K_NK; k++) {
        out->ms[k] = B->kms[k];
        out->launches[k] = B->klaunch[k];
        out->names[k] = kKernelNames[k];
    }
    return UG_OK;
}

int ug_batch_counters(void* h, int64_t* launches, int64_t* h2d_bytes, int64_t* d2h_bytes) {
    Batch* B = (Batch*)h;
    if (!B) return fail(UG_EINVAL, "null handle");
    if (launches) *launches = B->launches;
    if (h2d_bytes) *h2d_bytes = B->h2d;
    if (d2h_bytes) *d2h_bytes = B->d2h;
    return UG_OK;
}

int ug_batch_reset_times(void* h) {
    Batch* B = (Batch*)h;
    if (!B) return fail(UG_EINVAL, "bad arguments");
    for (int k = 0; k < K_NK; k++) {
        B->kms[k] = 0;
        B->klaunch[k] = 0;
    }
    return UG_OK;
}

int ug_batch_mixed_error(void* h, int32_t u, int64_t first, int64_t count, double* max_err, double* margin,
                         double* max_ratio) {
    Batch* B = (Batch*)h;
    if (!B || u < 0 || u >= B->n) return fail(UG_EINVAL, "bad arguments");
    if (B->opts.precision != UG_PREC_MIXED) return fail(UG_ENOTSUP, "batch is not mixed precision");
    return mixed_error(B->dU, u, B->U[u].d, B->U[u].mt, first, count, max_err, margin, max_ratio, B->st);
}

int ug_batch_destroy(void* h) {
    Batch* B = (Batch*)h;
    if (!B) return UG_OK;
    if (B->st) cudaStreamSynchronize(B->st);
    if (B->gexec) cudaGraphExecDestroy(B->gexec);
    for (UniHost& u : B->U) {
        for (void* p : u.owned) cudaFree(p);
        if (u.d.grid_kind == GRID_HASH) cudaFree(u.d.hslot);
        cudaFree(u.d.pts);
        cudaFree(u.d.ptf);
        cudaFree(u.d.acc_idx);
        mixed_free(u.mt);
    }
    cudaFree(B->dU);
    cudaFree(B->dCtl);
    cudaFree(B->d_gather_idx);
    cudaFree(B->d_gather_gid);
    cudaFree(B->d_gather_off);
    cudaFree(B->dInfo);
    for (int k = 0; k < 2 * K_NK; k++)
        if (B->ev[k]) cudaEventDestroy(B->ev[k]);
    if (B->own_stream && B->st) cudaStreamDestroy(B->st);
    delete B;
    return UG_OK;
}

int ug_pack_create(const ug_universe_cfg* cfg, const ug_run_opts* opts, void** out) {
    return ug_batch_create(cfg, 1, opts, out);
}
int ug_pack_run(void* h) { return ug_batch_run(h, 0); }
int ug_pack_stats(void* h, ug_stats* out) { return ug_batch_stats(h, 0, out); }
int ug_pack_destroy(void* h) { return ug_batch_destroy(h); }

}  // extern "C"
