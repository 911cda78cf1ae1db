// ug_mixed.cu -- tensor-core prefilter of the RSA packer (sm_100a).
//
// Position evaluation is a contraction: for a tile of 128 candidates and one
// axis,  D[m, n] = sum_k A[m, k] B[n, k]  with
//   A[m, .] = unnormalised coefficients of candidate m, three per frequency
//             pair p: (E_2p cos f / 2p, E_2p sin f / 2p, E_2p+1 / (2p+1)),
//             signs folded in, generated in FP32 straight into shared memory;
//   B[n, .] = (S_2p,t, Cm_2p,t, S_2p+1,t) / sin z_t for timestep t = order[n],
//             an FP64 host table split into BF16 hi + lo.
// The comoving position is X = wrap(D / sum_b E_b + a2).  A is split into
// BF16 hi + lo as well and the product runs as three tcgen05.mma passes
// (hi*hi + hi*lo + lo*hi) accumulating in FP32 in tensor memory.  The
// epilogue reads D with tcgen05.ld and runs the Chebyshev test against the
// FP32 copy of the collision grid with a guard band: a contact deeper than
// the band rejects, a separation wider than the band clears, anything in
// between marks the candidate for the FP64 retest (k_confirm64), so every
// decision equals the FP64 one.
//
// Pipeline per CTA (128 threads, one candidate per thread, persistent over
// tiles): shared memory holds two stages of {A_hi, A_lo, B_hi, B_lo}.  All
// threads generate stage s while the tensor core consumes stage s^1; one
// thread issues cp.async.bulk for the B chunk (completion on an mbarrier)
// and the MMAs (completion via tcgen05.commit on an mbarrier).  Every wait is
// bounded; on timeout the kernel records UG_ETIMEDOUT in the control block,
// frees its tensor memory and returns.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "ug_mixed.cuh"

namespace ug {

constexpr int kPairsPerChunk = 16;
constexpr int kKC = 3 * kPairsPerChunk;          // 48 coefficient entries per chunk
constexpr int kAImgBytes = kTile * kKC * 2;      // one BF16 A image (hi or lo)

// ------------------------------------------------------------ PTX helpers

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ uint64_t globaltimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Bounded wait: gives up after limit_ns of device time (or 2^26 polls).
__device__ __forceinline__ bool mbar_wait_ns(uint64_t* bar, uint32_t parity, uint64_t limit_ns) {
    if (mbar_try(bar, parity)) return true;
    const uint64_t t0 = globaltimer();
    for (uint32_t it = 0; it < (1u << 26); it++) {
        if (mbar_try(bar, parity)) return true;
        if ((it & 255) == 0 && globaltimer() - t0 > limit_ns) break;
    }
    return false;
}
// The prefilter's waits: ~1 s.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    return mbar_wait_ns(bar, parity, 1000000000ull);
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tmem_alloc(uint32_t* holder, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(holder)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
// D[tmem] (+)= A[smem] * B[smem]^T, BF16 inputs, FP32 accumulate, K = 16.
__device__ __forceinline__ void umma_bf16(uint32_t dtm, uint64_t ad, uint64_t bd, uint32_t idesc,
                                          uint32_t accum) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(dtm),
        "l"(ad), "l"(bd), "r"(idesc), "r"(accum)
        : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float* v) {
    uint32_t r[8];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 8; i++) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Shared-memory matrix descriptor, K-major, no swizzle: 8-row x 16-byte core
// matrices; lbo = byte stride between core matrices along K, sbo = along M/N.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// Instruction descriptor: kind::f16, BF16 x BF16 -> F32, both K-major.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// ---------------------------------------------------------- generation

// 1/b rounded to nearest FP32 (the value __frcp_rn gives), b = 0 .. kMaxF + 1;
// the frequency of a generation step is warp-uniform, so reads broadcast.
__constant__ float c_rcp[kMaxF + 2];

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&v);
}

// Coefficients of a quarter of one K chunk (pairs 4*part .. 4*part+3 of the
// chunk's 16) of candidate idx, axis ax, written as BF16 hi/lo into the rows
// of the canonical A images (12 entries = three 8-byte pieces per image).
// Returns the quarter's contribution to sum_b E_b.
__device__ __forceinline__ double gen_quarter(const UniDev& d, uint64_t idx, int ax, int ch, int part,
                                              bool valid, uint8_t* a_hi, uint8_t* a_lo, int row,
                                              double* sum_eb) {
    const int F = d.F;
    const int P = F >> 1;
    float v[12];
    double sum = 0.0, seb = 0.0;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int p = ch * kPairsPerChunk + part * 4 + q + 1;
        float ae = 0.f, be = 0.f, ao = 0.f;
        if (valid && p <= P) {
            const uint4 o = philox_block(d.seed, idx, ax, p);
            const float Ee = -__logf(((float)o.x + 0.5f) * 2.3283064365386963e-10f);
            const float f = (float)(o.z >> 1) * 4.656612873077393e-10f * 3.14159265358979f;
            float sf, cf;
            __sincosf(f, &sf, &cf);
            const float re = c_rcp[2 * p];
            const float we = Ee * re;
            const float se = (o.z & 1u) ? -we : we;
            ae = se * cf;
            be = se * sf;
            sum += (double)Ee;
            seb += (double)we;  // FP32 rounding of E_b / b is covered by the 1% slack of the band
            if (2 * p + 1 <= F) {
                const float Eo = -__logf(((float)o.y + 0.5f) * 2.3283064365386963e-10f);
                const float wo = Eo * c_rcp[2 * p + 1];
                ao = (o.w & 1u) ? -wo : wo;
                sum += (double)Eo;
                seb += (double)wo;
            }
        }
        v[3 * q] = ae;
        v[3 * q + 1] = be;
        v[3 * q + 2] = ao;
    }
#pragma unroll
    for (int g = 0; g < 3; g++) {
        uint32_t h[2], l[2];
#pragma unroll
        for (int e = 0; e < 2; e++) {
            const float x0 = v[4 * g + 2 * e], x1 = v[4 * g + 2 * e + 1];
            const __nv_bfloat16 h0 = __float2bfloat16_rn(x0), h1 = __float2bfloat16_rn(x1);
            h[e] = pack_bf16x2(__bfloat162float(h0), __bfloat162float(h1));
            l[e] = pack_bf16x2(x0 - __bfloat162float(h0), x1 - __bfloat162float(h1));
        }
        const int ent = part * 12 + 4 * g;  // first of 4 entries, never straddles an 8-entry core row
        const int off = (ent >> 3) * (kTile * 16) + row * 16 + (ent & 7) * 2;
        *reinterpret_cast<uint2*>(a_hi + off) = make_uint2(h[0], h[1]);
        *reinterpret_cast<uint2*>(a_lo + off) = make_uint2(l[0], l[1]);
    }
    *sum_eb += seb;
    return sum;
}

// ------------------------------------------------- guard-band grid test

// Group round, certain contact with point p at timestep t: joins the row to the
// point's group (*grp, shared by the row's threads).  True when the row already
// holds a different group (two groups touched: rejected).  Out of line: it is
// rare and keeps the neighbour scans small.
__device__ __noinline__ bool group_contact(const UniDev& d, int32_t p, int t, int* grp) {
    const int32_t gq = __ldg(&d.pts[UG_IDX((int64_t)p * d.T + t, d.slot_cap * d.T)].gid);
    int cur = *(volatile int*)grp;
    if (cur == -1) cur = atomicCAS(grp, -1, gq);
    return cur != -1 && cur != gq;
}

// FP32 Chebyshev test of X (dim coords) at timestep t against the committed
// packing.  Returns 1 when the candidate is certainly rejected; sets *gray when
// a pair lies in the guard band.  The cell range covers every point within
// r + m of X.  Group rounds (grp != nullptr): a certain contact joins the
// candidate to the contact's group in *grp (shared by the row's threads); a
// certain contact with a second group rejects.
template <int D, bool kEuclid, bool kCheckL1 = true>
__device__ __forceinline__ int test32_d(const UniDev& d, int t, const float* X, float r, float m,
                                        float inv_cell, int64_t cpt, bool* gray, int* grp, int* nvis) {
    // L2 ball: the FP32 distance vector is within sqrt(D) m of the exact one; r 1e-6
    // more covers the FP32 rounding of the squared sums compared below (relative
    // 3 2^-24 each).  The cell range covers the cube of half-width r + that bound.
    const float mE = kEuclid ? m * (D == 3 ? 1.7320508f : (D == 2 ? 1.4142136f : 1.0f)) * 1.001f + r * 1e-6f : m;
    const float band = mE * inv_cell + 1e-4f;
    int c[D], elo[D], ehi[D];
    float fr[D];
#pragma unroll
    for (int ax = 0; ax < D; ax++) {
        const float u = (X[ax] + 1.0f) * inv_cell;
        const float fl = floorf(u);
        fr[ax] = u - fl;
        int cc = (int)fl;
        c[ax] = cc >= d.gw ? d.gw - 1 : (cc < 0 ? 0 : cc);
    }
    // the neighbourhood below lies within 2 cells of c on every axis
    if (kCheckL1 && !occ1_hit<D>(d, t, c)) return 0;
#pragma unroll
    for (int ax = 0; ax < D; ax++) {
        elo[ax] = fr[ax] < band ? 1 : 0;
        ehi[ax] = fr[ax] > 1.0f - band ? 1 : 0;
    }
    Nbhd<D> nb;
    nbhd_make<D>(d, c, elo, ehi, nb);
    const float rin = r - mE, rout = r + mE;
    const float rin2 = rin > 0.f ? rin * rin : -1.f, rout2 = rout * rout;
    bool g = false;
    const bool deep = nbhd_scan<D>(d, t, nb, cpt, [&](int32_t p, int32_t& nx) -> bool {
        const uint4 qr = __ldg(reinterpret_cast<const uint4*>(d.ptf) + UG_IDX((int64_t)p * d.T + t, d.slot_cap * d.T));
        Pt32 q;
        q.c[0] = __uint_as_float(qr.x);
        q.c[1] = __uint_as_float(qr.y);
        q.c[2] = __uint_as_float(qr.z);
        q.next = (int32_t)qr.w;
        nx = q.next;
        ++*nvis;
        bool miss = false, in = true;
        if (kEuclid) {
            float s2 = 0.f;
#pragma unroll
            for (int ax = 0; ax < D; ax++) {
                const float dd = torus_deltaf(X[ax] - q.c[ax]);
                s2 = fmaf(dd, dd, s2);
            }
            miss = s2 > rout2;
            in = s2 < rin2;
        } else {
#pragma unroll
            for (int ax = 0; ax < D; ax++) {
                const float dd = fabsf(torus_deltaf(X[ax] - q.c[ax]));
                miss |= dd > rout;
                in &= dd < rin;
            }
        }
        if (miss) return false;
        if (in) return grp ? group_contact(d, p, t, grp) : true;
        g = true;
        return false;
    });
    if (g) *gray = true;
    return deep ? 1 : 0;
}

template <bool kEuclid, bool kCheckL1 = true>
__device__ __forceinline__ int test32_at(const UniDev& d, int t, const float* X, float r, float m,
                                         float inv_cell, int64_t cpt, bool* gray, int* grp, int* nvis) {
    if (d.dim == 3) return test32_d<3, kEuclid, kCheckL1>(d, t, X, r, m, inv_cell, cpt, gray, grp, nvis);
    if (d.dim == 2) return test32_d<2, kEuclid, kCheckL1>(d, t, X, r, m, inv_cell, cpt, gray, grp, nvis);
    return test32_d<1, false, kCheckL1>(d, t, X, r, m, inv_cell, cpt, gray, grp, nvis);  // 1 axis: ball == cube
}

// --------------------------------------------------------------- kernel

struct MixedLaunch {
    uint32_t ncols;    // tensor-memory columns per CTA
    int tpad_max;      // widest B image (rows) of the batch: sizes the B stage
    // debug dump of X (FP32 positions) for universe u, candidates [first, first+count),
    // and of the guard band of each (candidate, timestep)
    float* dump;
    float* dump_m;
    int u;
    int64_t first, count;
};

constexpr int kMxThreads = 512;  // 4 threads per candidate row
constexpr int kMxParts = kMxThreads / kTile;
constexpr int kXsFloats = 8 * 3 * 32 + 32 + 16;  // per-warp epilogue staging: positions, rho, columns
constexpr int kMxCompact = 24;
// the epilogue staging of all warps fits in the smallest pair of operand stages (T <= 16)
static_assert((kMxThreads / 32) * kXsFloats * 4 <= 2 * (2 * kAImgBytes + 16 * kKC * 2 * 2),
              "epilogue staging exceeds the operand stages");   // live rows of a warp at or below which their tests are spread (16, 24, 32 measured)

// kGroup: the batch holds group-mode universes (group rounds need the join /
// two-group logic in the neighbour scans; batches without them run without it).
// kEuclid: the batch holds universes with the L2-ball exclusion.
template <bool kGroup, bool kEuclid>
__global__ void __launch_bounds__(kMxThreads, 1) k_prefilter_mixed(const UniDev* __restrict__ U, UniCtl* ctl,
                                                                    RoundInfo* info, MixedLaunch L) {
    extern __shared__ __align__(1024) uint8_t sm[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // thread (row, part): warps w and w+4k share the tensor-memory lane quarter w%4
    const int row = (warp & 3) * 32 + lane;
    const int part = warp >> 2;
    // carve: two stages of {A_hi, A_lo, B (hi then lo)}; per-row state; barriers
    const int stage_bytes = 2 * kAImgBytes + L.tpad_max * kKC * 2 * 2;
    double* s_sum = reinterpret_cast<double*>(sm + 2 * stage_bytes);      // [kTile][kMxParts][2]
    int* s_rej = reinterpret_cast<int*>(s_sum + kTile * kMxParts * 2);   // [kTile]
    int* s_gray = s_rej + kTile;                                          // [kTile]
    int* s_grp = s_gray + kTile;                                          // [kTile] group rounds
    uint64_t* bar = reinterpret_cast<uint64_t*>(s_grp + kTile);
    uint64_t* bar_b = bar;       // [2] B chunk landed
    uint64_t* bar_m = bar + 2;   // [2] MMAs reading the stage finished
    uint64_t* bar_d = bar + 4;   // all MMAs of the pass finished
    uint32_t* holder = reinterpret_cast<uint32_t*>(bar + 5);

    // tile offsets of the universes, for the per-tile lookup of its universe
    __shared__ int32_t s_toff[kMaxUni + 1];
    if (L.dump == nullptr)
        for (int i = tid; i <= info->n_uni; i += blockDim.x) s_toff[i] = info->tile_off[i];
    if (warp == 0) tmem_alloc(holder, L.ncols);
    if (tid == 0) {
        for (int i = 0; i < 5; i++) mbar_init(&bar[i], 1);
        fence_mbar_init();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *holder;

    uint32_t ph_b[2] = {0, 0}, ph_m[2] = {0, 0}, ph_d = 0;
    int seq = 0;
    bool timeout = false;
    const bool dump = L.dump != nullptr;
    const int n_uni = dump ? 1 : info->n_uni;
    const int total = dump ? (int)((L.count + kTile - 1) / kTile) : info->total_tiles;
    volatile int* vrej = s_rej;
    volatile int* vgray = s_gray;

    // tiles: the first gridDim.x statically, the rest handed out one at a time
    // (tile costs differ by orders of magnitude across universes)
    // The next tile is claimed when a tile starts (its atomic's latency hides
    // behind the tile's work) into one of two slots read after the tile's last
    // barrier, so a slow reader never sees the slot overwritten.
    __shared__ int s_next[2];
    int npar = 0;
    auto next_tile = [&](int cur) -> int {
        if (dump) return cur + (int)gridDim.x;
        __syncthreads();
        const int nt = s_next[npar];
        npar ^= 1;
        return nt;
    };
    for (int tile = blockIdx.x; tile < total && !timeout; tile = next_tile(tile)) {
        if (!dump && tid == 0) s_next[npar] = (int)gridDim.x + atomicAdd(&info->tile_next, 1);
        const int pos = dump ? 0 : find_uni(s_toff, n_uni, tile);
        const int u = dump ? L.u : info->tile_uni[pos];
        const UniDev& d = U[u];
        const int lt = dump ? tile : tile - s_toff[pos];
        const uint64_t tile_t0 = tid == 0 ? globaltimer() : 0;
        const int off = lt * kTile + row;
        int64_t base;
        int B;
        if (dump) {
            base = L.first;
            B = (int)L.count;
        } else {
            base = ctl[u].round_base;
            B = ctl[u].B;
        }
        const bool valid = off < B;
        const uint64_t idx = (uint64_t)(base + off);
        if (!d.mx_ok) {  // not eligible for the tensor-core path: everything to the FP64 test
            if (part == 0) {
                const uint32_t g = __ballot_sync(0xffffffffu, valid);
                if (lane == 0 && !dump) {
                    d.surv_bits[UG_IDX(off >> 5, d.B_max / 32)] = 0u;
                    d.gray_bits[UG_IDX(off >> 5, d.B_max / 32)] = g;
                }
            }
            continue;
        }
        const int dim = d.dim, T = d.T, nch = d.mx_chunks, tpad = d.mx_tpad, nm = d.mx_nmma;
        const uint32_t bchunk = (uint32_t)tpad * kKC * 2 * 2;  // hi + lo images
        const uint32_t idesc = idesc_bf16(128, nm);
        const float r = (float)d.cell, mrg = d.mx_margin, inv_cell = (float)(1.0 / d.cell);
        const int64_t cpt = cells_per_t(d);
        const uint32_t* __restrict__ occ1 = d.occ1;
        const int gw = d.gw, occ1_gw = d.occ1_gw, occ1_sh = d.occ1_shift;
        const int64_t occ1_pt = d.occ1_per_t;
        // group semantics this round (unique-group mode, or phase 2 of the subpath mode)
        const bool group = kGroup && !dump &&
                           (d.group_mode == GROUP_UNIQUE || (d.group_mode == GROUP_SUBPATH && ctl[u].phase == 2));
        float inv_sum[3] = {0.f, 0.f, 0.f}, a2f[3] = {0.f, 0.f, 0.f};
        float rho = 0.f;  // largest sum_b (E_b / b) / sum E over the axes
        if (part == 0) {
            s_rej[row] = valid ? 0 : 1;
            s_gray[row] = 0;
            s_grp[row] = -1;
        }
        int nev = 0, nvis = 0;
        for (int pass = 0; pass < d.mx_npass && !timeout; pass++) {
            if (pass > 0 && __syncthreads_and(vrej[row] != 0)) break;
            for (int ax = 0; ax < dim && !timeout; ax++) {
                double sumE = 0.0, sumEb = 0.0;
                if (pass == 0 && valid) {
                    const uint4 o = philox_block(d.seed, idx, ax, 0);
                    const float v = d.pin ? 0.f : (float)((double)o.x * (1.0 / 2147483648.0) - 1.0);
#pragma unroll
                    for (int k = 0; k < 3; k++)  // selects: a dynamic index would go to local memory
                        if (k == ax) a2f[k] = v;
                }
                for (int ch = 0; ch < nch; ch++, seq++) {
                    const int st = seq & 1;
                    uint8_t* sbase = sm + st * stage_bytes;
                    uint8_t* a_hi = sbase;
                    uint8_t* a_lo = sbase + kAImgBytes;
                    uint8_t* b_img = sbase + 2 * kAImgBytes;
                    if (seq >= 2) {  // one thread polls; the CTA barrier releases the rest
                        if (tid == 0 && !mbar_wait(&bar_m[st], ph_m[st])) timeout = true;
                        ph_m[st] ^= 1;
                    }
                    if (__syncthreads_or(timeout)) {
                        timeout = true;
                        break;
                    }
                    if (tid == 0) {
                        mbar_expect_tx(&bar_b[st], bchunk);
                        bulk_g2s(b_img, d.mx_bimg + UG_IDX((int64_t)ch * bchunk + bchunk - 1, d.bimg_bytes) + 1 - bchunk,
                                 bchunk, &bar_b[st]);
                    }
                    sumE += gen_quarter(d, idx, ax, ch, part, valid, a_hi, a_lo, row, &sumEb);
                    fence_proxy_async();
                    __syncthreads();
                    if (tid == 0) {
                        if (!mbar_wait(&bar_b[st], ph_b[st])) timeout = true;
                        tc_fence_after();
                        if (!timeout) {
                            const uint32_t ah = smem_u32(a_hi), al = smem_u32(a_lo);
                            const uint32_t bh = smem_u32(b_img) + (uint32_t)(pass * nm * 16);
                            const uint32_t bl = bh + (uint32_t)tpad * kKC * 2;
                            const uint32_t dtm = tmem + (uint32_t)UG_IDX(ax * nm + nm - 1, L.ncols) + 1 - nm;
#pragma unroll
                            for (int j = 0; j < kKC / 16; j++) {
                                const uint64_t dah = sdesc(ah + j * 2 * (kTile * 16), kTile * 16, 128);
                                const uint64_t dal = sdesc(al + j * 2 * (kTile * 16), kTile * 16, 128);
                                const uint64_t dbh = sdesc(bh + j * 2 * (tpad * 16), tpad * 16, 128);
                                const uint64_t dbl = sdesc(bl + j * 2 * (tpad * 16), tpad * 16, 128);
                                umma_bf16(dtm, dah, dbh, idesc, (ch > 0 || j > 0) ? 1u : 0u);
                                umma_bf16(dtm, dah, dbl, idesc, 1u);
                                umma_bf16(dtm, dal, dbh, idesc, 1u);
                            }
                        }
                        umma_commit(&bar_m[st]);
                    }
                    ph_b[st] ^= 1;
                }
                if (timeout) break;
                if (pass == 0) {  // combine the four partial sums of the row in a fixed order
                    double* ss = s_sum + row * kMxParts * 2;
                    ss[2 * part] = sumE;
                    ss[2 * part + 1] = sumEb;
                    __syncthreads();
                    const double tot = ss[0] + ss[2] + ss[4] + ss[6];
                    const double teb = ss[1] + ss[3] + ss[5] + ss[7];
                    const float iv = valid ? (float)(1.0 / tot) : 0.f;
#pragma unroll
                    for (int k = 0; k < 3; k++)
                        if (k == ax) inv_sum[k] = iv;
                    if (valid) rho = fmaxf(rho, (float)(teb / tot));
                    __syncthreads();
                }
            }
            if (timeout) break;
            if (tid == 0) {
                umma_commit(bar_d);
                if (!mbar_wait(bar_d, ph_d)) timeout = true;
            }
            ph_d ^= 1;
            if (__syncthreads_or(timeout)) {
                timeout = true;
                break;
            }
            tc_fence_after();
            if (dim == 1 && d.cross1d && !dump) {
                // 1+1D with the crossing rule: stage the FP32 trajectory (natural
                // timestep order; the stages are free once the MMAs are done), then
                // test every accepted path at every timestep.
                float* xs = reinterpret_cast<float*>(sm);
                const int pitch = T + 1;
                const uint32_t lb = tmem + ((uint32_t)((warp & 3) * 32) << 16);
                for (int c0 = part * 8; c0 < nm; c0 += 8 * kMxParts) {
                    float x8[8];
                    tmem_ld8(lb + (uint32_t)UG_IDX(c0 + 7, L.ncols) - 7, x8);
                    tmem_wait_ld();
                    for (int j = 0; j < 8; j++)
                        if (c0 + j < T) xs[row * pitch + c0 + j] = torus_wrapf(fmaf(x8[j], inv_sum[0], a2f[0]));
                }
                tc_fence_before();
                __syncthreads();
                const int64_t ns = ctl[u].n_slots;
                const float rin = r - mrg, rout = r + mrg;
                // walk of one accepted path: every timestep up to the first certain contact
                auto walk = [&](int64_t sl) {
                    const Pt32* q = d.ptf + UG_IDX(sl * T + T - 1, d.slot_cap * T) + 1 - T;
                    bool hit = false, g = false;
                    float d0 = torus_deltaf(xs[row * pitch] - __ldg(&q[0].c[0]));
                    float a0 = fabsf(d0);
                    hit = a0 < rin;
                    g = !hit && a0 <= rout;
                    // the path's points 8 timesteps at a time: 8 independent loads in flight
                    for (int t0 = 1; t0 < T && !hit; t0 += 8) {
                        if (vrej[row]) break;  // another part of the row found a contact
                        float qv[8];
#pragma unroll
                        for (int k = 0; k < 8; k++) qv[k] = t0 + k < T ? __ldg(&q[t0 + k].c[0]) : 0.f;
#pragma unroll
                        for (int k = 0; k < 8; k++) {
                            if (hit || t0 + k >= T) break;
                            const float d1 = torus_deltaf(xs[row * pitch + t0 + k] - qv[k]);
                            const float a1 = fabsf(d1);
                            if (a1 < rin) {
                                hit = true;
                                break;
                            }
                            g = g || a1 <= rout;
                            // crossing: certain when both signs are certain and the sum is clear of 1
                            const bool flip = (d0 < 0.f) != (d1 < 0.f);
                            const bool signs_sure = a0 > mrg && a1 > mrg;
                            const float sum = a0 + a1;
                            if (flip && signs_sure && sum < 1.f - 2.f * mrg) {
                                hit = true;
                                break;
                            }
                            if ((!signs_sure && sum < 1.f + 2.f * mrg) ||
                                (flip && sum >= 1.f - 2.f * mrg && sum <= 1.f + 2.f * mrg))
                                g = true;
                            d0 = d1;
                            a0 = a1;
                        }
                    }
                    nev += T;
                    if (hit) vrej[row] = 1;
                    else if (g) vgray[row] = 1;
                };
                // The paths are walked nearest first: a candidate that meets any path
                // almost always meets one of the two paths beside it at the first
                // timestep (those lie between it and every other path) first.  Each
                // part finds the nearest path below and above among its slots; the
                // row's four parts combine them through the (idle) partial-sum array.
                float blo = 4.f, bhi = 4.f;  // distances below / above
                int slo = -1, shi = -1;
                if (!vrej[row]) {
                    const float x0 = xs[row * pitch];
                    for (int64_t sl = part; sl < ns; sl += kMxParts) {
                        const float dd = torus_deltaf(x0 - __ldg(&d.ptf[UG_IDX(sl * T, d.slot_cap * T)].c[0]));
                        if (dd >= 0.f) {
                            if (dd < blo) blo = dd, slo = (int)sl;
                        } else if (-dd < bhi) {
                            bhi = -dd, shi = (int)sl;
                        }
                    }
                }
                float* nbv = reinterpret_cast<float*>(s_sum);        // [kTile][kMxParts][2]
                int* nbs = reinterpret_cast<int*>(nbv + kTile * kMxParts * 2);
                nbv[(row * kMxParts + part) * 2] = blo;
                nbv[(row * kMxParts + part) * 2 + 1] = bhi;
                nbs[(row * kMxParts + part) * 2] = slo;
                nbs[(row * kMxParts + part) * 2 + 1] = shi;
                __syncthreads();
                blo = bhi = 4.f;  // same scan in every part: the same pair, ties to the lower part
                slo = shi = -1;
#pragma unroll
                for (int p2 = 0; p2 < kMxParts; p2++) {
                    const float vl = nbv[(row * kMxParts + p2) * 2], vh = nbv[(row * kMxParts + p2) * 2 + 1];
                    if (vl < blo) blo = vl, slo = nbs[(row * kMxParts + p2) * 2];
                    if (vh < bhi) bhi = vh, shi = nbs[(row * kMxParts + p2) * 2 + 1];
                }
                // every part now holds the same pair: parts 0 and 1 walk it, then
                // (rows still alive) all parts walk their own slots but those two
                if (part == 0 && slo >= 0 && !vrej[row]) walk(slo);
                if (part == 1 && shi >= 0 && !vrej[row]) walk(shi);
                __syncthreads();
                for (int64_t sl = part; sl < ns; sl += kMxParts) {
                    if (vrej[row]) break;
                    if (sl == slo || sl == shi) continue;
                    walk(sl);
                }
                __syncthreads();
                continue;  // single pass for dim 1
            }
            // epilogue: 8-column blocks part, part+4, ... of this pass (endpoint-first order)
            const uint32_t lane_base = tmem + ((uint32_t)((warp & 3) * 32) << 16);
            for (int c0 = part * 8; c0 < nm; c0 += 8 * kMxParts) {
                const int col0 = pass * nm + c0;
                if (col0 >= T) break;
                if (!dump && __all_sync(0xffffffffu, vrej[row] != 0)) break;
                float x[3][8];
#pragma unroll
                for (int ax = 0; ax < 3; ax++)
                    if (ax < dim) tmem_ld8(lane_base + (uint32_t)UG_IDX(ax * nm + c0 + 7, L.ncols) - 7, x[ax]);
                tmem_wait_ld();
                if (dump) {
                    for (int j = 0; j < 8; j++) {
                        const int col = col0 + j;
                        if (col >= T) break;
                        // the crossing rule's B image (1+1D) holds the timesteps in natural order
                        const int t = (dim == 1 && d.cross1d) ? col : __ldg(d.order + col);
                        // guard band of this timestep (1% over the bound: FP32 evaluation of it)
                        const float bnd = fminf(2.f, 2.f * (float)__ldg(d.invsinz + t) * rho);
                        const float mt = (2.f * d.mx_mc1 * bnd + d.mx_mc0) * 1.01f;
                        if (valid) {
                            for (int ax = 0; ax < dim; ax++)
                                L.dump[((size_t)off * T + t) * dim + ax] =
                                    torus_wrapf(fmaf(x[ax][j], inv_sum[ax], a2f[ax]));
                            L.dump_m[(size_t)off * T + t] = mt;
                        }
                    }
                    continue;
                }
                const uint32_t am = __ballot_sync(0xffffffffu, valid && !vrej[row]);
                const int na = __popc(am);
                if (na == 0) continue;
                const int ncol = min(8, T - col0);
                // The block's work is its (live row, column) tests.  Many live rows: each
                // lane tests its own row's columns.  Few (<= kMxCompact): the tests are
                // spread over all 32 lanes, column-major, so dead rows leave no lane idle.
                // Either way a lane first issues the first-level loads of all its tests
                // together (the dilated occupancy bit of each test point's own cell
                // block; a clear bit proves the neighbourhood empty), then runs the
                // exact test only where a bit is set.  The block's positions and column
                // data are staged in this warp's slice of the (now idle) operand stages.
                float* xs = reinterpret_cast<float*>(sm) + warp * kXsFloats;  // [8][3][32], rho[32], t[8], isz[8]
                int* xt = reinterpret_cast<int*>(xs + 8 * 3 * 32 + 32);
                float* xz = xs + 8 * 3 * 32 + 32 + 8;
                if (lane < ncol) {
                    const int t = __ldg(d.order + col0 + lane);
                    xt[lane] = t;
                    xz[lane] = (float)__ldg(d.invsinz + t);
                }
#pragma unroll
                for (int j = 0; j < 8; j++)
#pragma unroll
                    for (int ax = 0; ax < 3; ax++)
                        if (j < ncol && ax < dim)
                            xs[(j * 3 + ax) * 32 + lane] = torus_wrapf(fmaf(x[ax][j], inv_sum[ax], a2f[ax]));
                xs[8 * 3 * 32 + lane] = rho;
                __syncwarp();
                const bool spread = na <= kMxCompact;
                const int nitems = spread ? na * ncol : (((am >> lane) & 1u) ? ncol : 0);
                const int rbase = (warp & 3) * 32;
                uint32_t wv[8];
                uint64_t bsh = 0;  // bit position of each test's block in its word, 5 bits each
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    const int i = spread ? lane + 32 * k : k;
                    wv[k] = 0u;
                    if (i < nitems) {
                        const int j = spread ? i / na : k;
                        const int src = spread ? (int)__fns(am, 0, i - j * na + 1) : lane;
                        const int t = xt[j];
                        int64_t lin = 0;
#pragma unroll
                        for (int ax = 0; ax < 3; ax++) {
                            if (ax >= dim) break;
                            int cc = (int)floorf((xs[(j * 3 + ax) * 32 + src] + 1.0f) * inv_cell);
                            cc = cc >= gw ? gw - 1 : (cc < 0 ? 0 : cc);
                            lin = lin * occ1_gw + (cc >> occ1_sh);
                        }
                        const int64_t b = (int64_t)t * occ1_pt + lin;
                        bsh |= (uint64_t)(b & 31) << (5 * k);
                        wv[k] = __ldg(occ1 + (b >> 5));
                    }
                }
                uint32_t need = 0;
#pragma unroll
                for (int k = 0; k < 8; k++) need |= ((wv[k] >> ((bsh >> (5 * k)) & 31)) & 1u) << k;
                // tests of this lane (main: the row's columns up to its first certain contact)
                int tested = spread ? (nitems > lane ? (nitems - lane + 31) / 32 : 0) : nitems;
                while (need) {
                    const int k = __ffs(need) - 1;
                    need &= need - 1;
                    const int i = spread ? lane + 32 * k : k;
                    const int j = spread ? i / na : k;
                    const int src = spread ? (int)__fns(am, 0, i - j * na + 1) : lane;
                    const int rrow = rbase + src;
                    if (vrej[rrow]) {
                        if (!spread) {
                            tested = k;
                            break;
                        }
                        continue;
                    }
                    const int t = xt[j];
                    float X[3];
#pragma unroll
                    for (int ax = 0; ax < 3; ax++) X[ax] = ax < dim ? xs[(j * 3 + ax) * 32 + src] : 0.f;
                    // guard band of this timestep (1% over the bound: FP32 evaluation of it)
                    const float bnd = fminf(2.f, 2.f * xz[j] * xs[8 * 3 * 32 + src]);
                    const float mt = (2.f * d.mx_mc1 * bnd + d.mx_mc0) * 1.01f;
                    bool gr = false;
                    int* gp = (kGroup && group) ? s_grp + rrow : nullptr;
                    const int dead = (kEuclid && d.euclid)
                                         ? test32_at<true, false>(d, t, X, r, mt, inv_cell, cpt, &gr, gp, &nvis)
                                         : test32_at<false, false>(d, t, X, r, mt, inv_cell, cpt, &gr, gp, &nvis);
                    if (gr) vgray[rrow] = 1;
                    if (dead) {
                        vrej[rrow] = 1;
                        if (!spread) {
                            tested = k + 1;
                            break;
                        }
                    }
                }
                nev += tested;
                __syncwarp();
            }
            tc_fence_before();
            __syncthreads();
        }
        if (!dump) {
            for (int o = 16; o > 0; o >>= 1) nev += __shfl_xor_sync(0xffffffffu, nev, o);
            for (int o = 16; o > 0; o >>= 1) nvis += __shfl_xor_sync(0xffffffffu, nvis, o);
            if (lane == 0 && nev) atomicAdd((unsigned long long*)&ctl[u].evals, (unsigned long long)nev);
            if (lane == 0 && nvis) atomicAdd((unsigned long long*)&ctl[u].visits, (unsigned long long)nvis);
            if (part == 0) {
                const bool rej = vrej[row] != 0, gry = vgray[row] != 0;
                const bool surv = valid && !rej && !gry && !timeout;
                const bool gr = valid && !rej && (gry || timeout);
                const uint32_t sb = __ballot_sync(0xffffffffu, surv);
                const uint32_t gb = __ballot_sync(0xffffffffu, gr);
                if (kGroup && surv && d.group_mode != GROUP_NONE) d.g0[UG_IDX(off, d.B_max)] = s_grp[row];
                if (lane == 0) {
                    d.surv_bits[UG_IDX(off >> 5, d.B_max / 32)] = sb;
                    d.gray_bits[UG_IDX(off >> 5, d.B_max / 32)] = gb;
                    const int ng = __popc(gb);
                    if (ng) atomicAdd((unsigned long long*)&ctl[u].gray_total, (unsigned long long)ng);
                }
            }
            if (tid == 0) {  // this tile's time orders the next round's tiles
                const uint64_t dt = globaltimer() - tile_t0;
                atomicMax(&ctl[u].tile_ns, (int)(dt < 0x7fffffffull ? dt : 0x7fffffffull));
            }
            __syncthreads();
        }
    }
    if (timeout && tid == 0 && !dump) {
        for (int v = 0; v < n_uni; v++) {
            ctl[v].err_code = UG_ETIMEDOUT;
            ctl[v].state = ST_ERROR;
        }
    }
    // drain: the last commits of this CTA must land before tensor memory is freed
    if (tid == 0 && seq > 0) {
        const int s1 = (seq - 1) & 1;
        mbar_wait(&bar_m[s1], ph_m[s1]);
        if (seq > 1) mbar_wait(&bar_m[s1 ^ 1], ph_m[s1 ^ 1]);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) tmem_dealloc(tmem, L.ncols);
}

// Self-test of the bounded wait: one thread waits on an mbarrier that nothing
// arrives on.  The wait gives up after limit_ns and the kernel records
// UG_ETIMEDOUT in *status and returns, as the prefilter does on a stuck pipeline.
__global__ void k_wait_selftest(uint64_t limit_ns, int32_t* status) {
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) *status = mbar_wait_ns(&bar, 0, limit_ns) ? UG_OK : UG_ETIMEDOUT;
}

int wait_selftest(int64_t limit_ns, int32_t* status) {
    int32_t* d = nullptr;
    if (cudaMalloc(&d, sizeof(int32_t)) != cudaSuccess) return UG_ENOMEM;
    cudaMemset(d, 0xff, sizeof(int32_t));
    k_wait_selftest<<<1, 32>>>((uint64_t)limit_ns, d);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(status, d, sizeof(int32_t), cudaMemcpyDeviceToHost);
    cudaFree(d);
    return e == cudaSuccess ? UG_OK : UG_ECUDA;
}

// FP64 positions of candidates [first, first+count) (Philox stream) for the
// achieved-error measurement.
__global__ void k_pos64(const UniDev* __restrict__ U, int u, int64_t first, int64_t count, double* out) {
    const UniDev& d = U[u];
    double alpha[3 * (kMaxF + 1)], beta[3 * (kMaxF + 1)], a2[3];
    const int F1 = d.F + 1;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count;
         i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t idx = (uint64_t)(first + i);
        for (int ax = 0; ax < d.dim; ax++) a2[ax] = gen_philox64(d, idx, ax, alpha + ax * F1, beta + ax * F1, 1);
        for (int t = 0; t < d.T; t++)
            for (int ax = 0; ax < d.dim; ax++)
                out[((size_t)i * d.T + t) * d.dim + ax] = eval64(d, alpha + ax * F1, beta + ax * F1, 1, a2[ax], t);
    }
}

// ------------------------------------------------------------------ host

static int g_ncols = 32;
static int g_tpad_max = 16;
static size_t g_smem = 0;
static int g_ctas_per_sm = 1;

static size_t smem_bytes() {
    return (size_t)2 * (2 * kAImgBytes + g_tpad_max * kKC * 2 * 2) + (size_t)kTile * kMxParts * 16 +
           3 * kTile * 4 + 64;
}

static uint16_t bf16_bits(float x) {
    const __nv_bfloat16 h = __float2bfloat16_rn(x);
    return *reinterpret_cast<const uint16_t*>(&h);
}
static float bf16_val(uint16_t b) {
    uint32_t u = (uint32_t)b << 16;
    float f;
    memcpy(&f, &u, 4);
    return f;
}

int mixed_setup(const ug_universe_cfg& cfg, UniDev& d, MixedTables& mt) {
    const int T = cfg.T, F = cfg.T, dim = cfg.dim;
    // group rounds of the 1+1D crossing rule stay on the FP64 path
    d.mx_ok = (cfg.rng == UG_RNG_PHILOX && !(cfg.cross1d && cfg.group_mode != UG_GROUP_NONE)) ? 1 : 0;
    const bool natural = cfg.dim == 1 && cfg.cross1d;  // the crossing test walks t in order
    const int P = F / 2;
    const int nch = (P + kPairsPerChunk - 1) / kPairsPerChunk;
    // B rows: timesteps padded to 16; when dim * rows exceeds the 512 tensor
    // memory columns, two passes of exactly half the (32-padded) rows each
    int tpad = (T + 15) / 16 * 16;
    int nm = tpad, npass = 1;
    if (dim * tpad > 512) {
        tpad = (T + 31) / 32 * 32;
        nm = tpad / 2;
        npass = 2;
    }
    d.mx_chunks = nch;
    d.mx_tpad = tpad;
    d.mx_nmma = nm;
    d.mx_npass = npass;
    // guard band: split-BF16 product error 3 * 2^-16 * sum|A||B| with
    // sum|A||B| / sum E <= 2 (|sin bz| <= b sin z, |cos bz - 1| <= b sin z for even b),
    // FP32 accumulation of 3K products (<= 2^-23 each, relative to the same sum),
    // FP32 generation (logf, sincosf, reciprocals: < 2e-6), stored FP32 points and
    // the FP32 subtraction (< 4e-7); doubled for safety.
    // The bound 2 on sum|A||B| / sum E tightens per candidate and timestep to
    // min(2, 2 rho / sin z_t): the pair terms of frequency b are at most
    // (E_b / b) * 2 / sin z_t (Cauchy-Schwarz over (cos f, sin f) with
    // |sin x|^2 + |cos x - 1|^2 <= 4), so their sum is at most
    // (2 / sin z_t) sum_b E_b / b = (2 / sin z_t) rho sum E.
    const int K = nch * kKC;
    const double mc1 = 3.0 * std::ldexp(1.0, -16) + 3.0 * K * std::ldexp(1.0, -23);
    const double mc0 = 2.0 * 2e-6 + 4e-7;
    const double m = 2.0 * mc1 * 2.0 + mc0;
    d.mx_margin = (float)m;
    // first-level filter reach: radius + the widest band a test applies (1.01 m,
    // sqrt(d) m + r 1e-6 for the L2 ball), with 2% and 1e-3 cell of slack for the
    // FP32 cell index of the test point
    d.occ1_reach = d.cell + 1.02 * m * (cfg.euclid ? std::sqrt((double)dim) * 1.001 : 1.0) +
                   (cfg.euclid ? d.cell * 1e-6 : 0.0) + d.cell * 1e-3;
    d.mx_mc1 = (float)mc1;
    d.mx_mc0 = (float)mc0;
    mt.margin = m;
    mt.K = K;
    mt.Tp = tpad;
    // B images
    std::vector<double> S((size_t)(F + 1) * T), Cm((size_t)(F + 1) * T), inv(T);
    std::vector<int32_t> order(T);
    {
        std::vector<double> z(T);
        for (int i = 0; i < T; i++) {
            z[i] = cfg.zgrid == UG_ZGRID_REF ? (i + 1) * kPi / (T + 1) : (i + 0.5) * kPi / T;
            inv[i] = 1.0 / sin(z[i]);
        }
        for (int b = 0; b <= F; b++)
            for (int t = 0; t < T; t++) {
                S[(size_t)b * T + t] = sin(b * z[t]);
                Cm[(size_t)b * T + t] = cos(b * z[t]) - 1.0;
            }
        for (int i = 0; i < T; i++) order[i] = i;
        if (!natural)
            std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
                return std::min(a, T - 1 - a) < std::min(b, T - 1 - b);
            });
    }
    const size_t img = (size_t)tpad * kKC;  // BF16 elements per hi (or lo) image
    std::vector<uint16_t> host((size_t)nch * 2 * img, 0);
    for (int ch = 0; ch < nch; ch++) {
        uint16_t* hi = host.data() + (size_t)ch * 2 * img;
        uint16_t* lo = hi + img;
        for (int kk = 0; kk < kKC; kk++) {
            const int p = ch * kPairsPerChunk + kk / 3 + 1, s = kk % 3;
            for (int n = 0; n < tpad; n++) {
                double v = 0.0;
                if (n < T && p <= P) {
                    const int t = order[n];
                    const int b = s == 2 ? 2 * p + 1 : 2 * p;
                    if (b <= F) v = (s == 1 ? Cm[(size_t)b * T + t] : S[(size_t)b * T + t]) * inv[t];
                }
                const uint16_t h = bf16_bits((float)v);
                const uint16_t l = bf16_bits((float)(v - (double)bf16_val(h)));
                const size_t e = (size_t)(kk / 8) * (tpad * 8) + (size_t)n * 8 + (kk % 8);
                hi[e] = h;
                lo[e] = l;
            }
        }
    }
    void* dimg = nullptr;
    if (cudaMalloc(&dimg, host.size() * 2) != cudaSuccess) return UG_ENOMEM;
    if (cudaMemcpy(dimg, host.data(), host.size() * 2, cudaMemcpyHostToDevice) != cudaSuccess) return UG_ECUDA;
    mt.bhi = dimg;
    d.mx_bimg = (const uint8_t*)dimg;
    d.bimg_bytes = (int64_t)host.size() * 2;
    // tensor-memory columns: the widest universe decides (power of two >= 32)
    if (tpad > g_tpad_max) g_tpad_max = tpad;
    int cols = dim * nm;
    int nc = 32;
    while (nc < cols) nc <<= 1;
    if (nc > g_ncols) g_ncols = nc;
    return UG_OK;
}

void mixed_free(MixedTables& mt) {
    if (mt.bhi) cudaFree(mt.bhi);
    mt.bhi = nullptr;
}

int mixed_init_kernels() {
    {
        float rcp[kMaxF + 2];
        rcp[0] = 0.f;
        for (int b = 1; b < kMaxF + 2; b++) rcp[b] = (float)(1.0 / (double)b);
        if (cudaMemcpyToSymbol(c_rcp, rcp, sizeof rcp) != cudaSuccess) return UG_ECUDA;
    }
    g_smem = smem_bytes();
    // UG_SMEM_PAD=1: request (nearly) all shared memory, one CTA per SM
    const char* pad = getenv("UG_SMEM_PAD");
    if (pad && pad[0] == '1') g_smem = std::max<size_t>(g_smem, 220 * 1024);
    // at most 512 / ncols CTAs per SM may hold tensor memory at once: pad the
    // shared-memory request so that no more than that many are resident
    const int by_tmem = 512 / g_ncols;
    int dev = 0, smem_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    size_t req = g_smem;
    const size_t per_cta_reserved = 1024;
    int fit = (int)(smem_sm / (req + per_cta_reserved));
    if (fit > by_tmem) req = smem_sm / (by_tmem + 1) - per_cta_reserved + 16;
    g_smem = std::max(req, g_smem);
    g_ctas_per_sm = std::max(1, std::min(by_tmem, (int)(smem_sm / (g_smem + per_cta_reserved))));
    if (cudaFuncSetAttribute(k_prefilter_mixed<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)g_smem) != cudaSuccess ||
        cudaFuncSetAttribute(k_prefilter_mixed<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)g_smem) != cudaSuccess ||
        cudaFuncSetAttribute(k_prefilter_mixed<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)g_smem) != cudaSuccess ||
        cudaFuncSetAttribute(k_prefilter_mixed<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)g_smem) != cudaSuccess)
        return UG_ECUDA;
    return UG_OK;
}

void launch_prefilter_mixed(const UniDev* dU, UniCtl* dCtl, RoundInfo* dInfo, int nsm, bool any_group,
                            bool any_euclid, cudaStream_t st) {
    MixedLaunch L{(uint32_t)g_ncols, g_tpad_max, nullptr, nullptr, 0, 0, 0};
    const int g = nsm * g_ctas_per_sm;
    if (any_group && any_euclid)
        k_prefilter_mixed<true, true><<<g, kMxThreads, g_smem, st>>>(dU, dCtl, dInfo, L);
    else if (any_group)
        k_prefilter_mixed<true, false><<<g, kMxThreads, g_smem, st>>>(dU, dCtl, dInfo, L);
    else if (any_euclid)
        k_prefilter_mixed<false, true><<<g, kMxThreads, g_smem, st>>>(dU, dCtl, dInfo, L);
    else
        k_prefilter_mixed<false, false><<<g, kMxThreads, g_smem, st>>>(dU, dCtl, dInfo, L);
}

int mixed_error(const UniDev* dU, int u, const UniDev& d, const MixedTables& mt, int64_t first, int64_t count,
                double* max_err, double* margin, double* max_ratio, cudaStream_t st) {
    if (!d.mx_ok) return UG_ENOTSUP;
    const size_t nm = (size_t)count * d.T;
    const size_t n = nm * d.dim;
    float *d32 = nullptr, *dm = nullptr;
    double* d64 = nullptr;
    if (cudaMalloc(&d32, n * 4) != cudaSuccess || cudaMalloc(&dm, nm * 4) != cudaSuccess ||
        cudaMalloc(&d64, n * 8) != cudaSuccess) {
        cudaFree(d32);
        cudaFree(dm);
        return UG_ENOMEM;
    }
    cudaMemsetAsync(d32, 0, n * 4, st);
    cudaMemsetAsync(dm, 0, nm * 4, st);
    MixedLaunch L{(uint32_t)g_ncols, g_tpad_max, d32, dm, u, first, count};
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, 0);
    k_prefilter_mixed<false, false><<<nsm * g_ctas_per_sm, kMxThreads, g_smem, st>>>(dU, nullptr, nullptr, L);
    k_pos64<<<(int)std::min<int64_t>((count + 127) / 128, 2048), 128, 0, st>>>(dU, u, first, count, d64);
    std::vector<float> h32(n), hm(nm);
    std::vector<double> h64(n);
    cudaError_t e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = cudaMemcpy(h32.data(), d32, n * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(hm.data(), dm, nm * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(h64.data(), d64, n * 8, cudaMemcpyDeviceToHost);
    cudaFree(d32);
    cudaFree(dm);
    cudaFree(d64);
    if (e != cudaSuccess) return UG_ECUDA;
    double mx = 0.0, ratio = 0.0;
    for (size_t i = 0; i < n; i++) {
        double df = fabs((double)h32[i] - h64[i]);
        df = std::min(df, 2.0 - df);
        mx = std::max(mx, df);
        const double band = (double)hm[i / d.dim];
        ratio = std::max(ratio, band > 0.0 ? df / band : INFINITY);
    }
    *max_err = mx;
    *margin = mt.margin;
    *max_ratio = ratio;
    return UG_OK;
}

}  // namespace ug
