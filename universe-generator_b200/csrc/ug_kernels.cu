// ug_kernels.cu -- the round pipeline of the batched RSA packer.
//
// One round of every active universe:
//   k_plan         round sizes, phase transitions, tile decomposition
//   k_gray_compact + k_confirm64w
//                  FP64 form: every candidate, warp per candidate (shared-memory
//                  coefficients, lanes over timesteps) against the committed packing;
//                  mixed form: k_prefilter_mixed (ug_mixed.cu), then the same warp
//                  test for the candidates its guard band left undecided
//   k_compact      survivors in candidate-index order (deterministic)
//   k_surv_gen     FP64 coefficients of the survivors (term-ordered rows)
//   k_surv_gemm    their FP64 trajectories as a register-tiled product
//   k_surv_hash    round-table insert of every survivor timestep
//   k_conflicts    each survivor's contacts with EARLIER survivors of the round
//   k_greedy       in-order resolution: survivor i is admitted iff it touches
//                  no admitted earlier survivor (group rules in group modes)
//   k_commit       admitted trajectories appended to the collision grid
// Non-survivors collide with the committed packing, which only grows, so they
// are rejected by sequential RSA as well; survivors are decided in index
// order against the round's earlier admissions.  The accepted set is
// therefore exactly sequential RSA over the candidate stream -- the
// exact-index admission of cuda/braid_knot.cu:433-462, made device-resident.
#include "ug_kernels.cuh"

#include <algorithm>

namespace ug {

// ------------------------------------------------------------------ plan

// Closes the bucket ending at phase position in_phase (a multiple of q) with the
// count cur; true when the phase stops there: 32 buckets, more than 1e6
// candidates decided, and the last 32 buckets' count / (32 q) below thr.
__device__ __forceinline__ bool win_close(int64_t q, int64_t& nb, int64_t& sum, int64_t& cur, int64_t* ring,
                                          double thr, int64_t in_phase) {
    if (q <= 0 || in_phase <= 0 || in_phase % q) return false;
    const int slot = (int)(nb & 31);
    if (nb >= 32) sum -= ring[slot];
    ring[slot] = cur;
    sum += cur;
    cur = 0;
    nb++;
    return nb >= 32 && in_phase > 1000000 && (double)sum / (double)(32 * q) < thr;
}

// Exclusive prefix of v over the 256 threads of the block; *total gets the sum.
// Every thread of the block must call it (it synchronises the block).
__device__ __forceinline__ int block_excl_scan256(int v, int* wsum, int* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int incl = v;
    for (int o = 1; o < 32; o <<= 1) {
        const int x = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += x;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    int wpre = 0, tot = 0;
    for (int k = 0; k < 8; k++) {
        if (k < warp) wpre += wsum[k];
        tot += wsum[k];
    }
    __syncthreads();  // wsum is reused by the next call
    *total = tot;
    return wpre + incl - v;
}

__global__ void k_plan(const UniDev* __restrict__ U, UniCtl* ctl, RoundInfo* info) {
    __shared__ int32_t ntiles[kMaxUni];
    __shared__ int32_t cost[kMaxUni];
    __shared__ int32_t order[kMaxUni];
    const int n = info->n_uni;
    for (int u = threadIdx.x; u < n; u += blockDim.x) {
        UniCtl& c = ctl[u];
        const UniDev& d = U[u];
        int B = 0;
        // tile cost: the last round's slowest prefilter tile; before any is timed,
        // dim * T stands in (all universes start together, so one round uses one kind)
        cost[u] = c.tile_ns > 0 ? c.tile_ns : d.dim * d.T;
        c.tile_ns = 0;
        // the last round's admissions (k_greedy) and newly occupied cells (k_commit)
        // close the windows' buckets; rounds end on bucket boundaries
        {
            const int64_t nc = c.round_new;
            c.round_new = 0;
            c.filled += nc;
            if (c.last_used > 0 && c.state == ST_ACTIVE) {
                const int64_t in_phase = c.next_cand - c.phase_start;
                c.win_cur += c.accepted_round;
                c.fwin_cur += nc;
                const bool sa = win_close(c.win_q, c.win_nb, c.win_sum, c.win_cur, c.win_ring, c.win_thr, in_phase);
                const bool sf = win_close(c.fwin_q, c.fwin_nb, c.fwin_sum, c.fwin_cur, c.fwin_ring, c.sub_fill_rate,
                                          in_phase);
                if (sa || sf) c.phase_end = c.next_cand;  // stops below
            }
            c.last_used = 0;
        }
        if (c.state == ST_ACTIVE) {
            for (int guard = 0; guard < 2; guard++) {
                const bool over = c.next_cand >= c.phase_end ||
                                  (c.phase == 1 && c.max_n > 0 && c.n_unique >= c.max_n);
                if (!over) break;
                if (c.phase == 1 && d.group_mode == GROUP_SUBPATH) {
                    c.phase = 2;
                    c.phase1_end = c.next_cand;
                    c.phase_start = c.next_cand;
                    c.phase_end = c.next_cand + c.sub_budget;
                    c.round_B = c.B_cap;  // fresh adaptation (braid_cuda.cu:952)
                    c.win_thr = c.sub_accept_rate;
                    c.win_q = win_bucket(c.sub_accept_rate);
                    c.win_nb = c.win_sum = c.win_cur = 0;
                    c.fwin_q = win_bucket(c.sub_fill_rate);
                    c.fwin_nb = c.fwin_sum = c.fwin_cur = 0;
                    continue;
                }
                c.state = ST_DONE;
                break;
            }
            if (c.state == ST_ACTIVE) {
                int64_t left = c.phase_end - c.next_cand;
                const int64_t in_phase = c.next_cand - c.phase_start;
                if (c.win_q > 0) left = min(left, c.win_q - in_phase % c.win_q);
                if (c.fwin_q > 0) left = min(left, c.fwin_q - in_phase % c.fwin_q);
                const int cap = c.round_B < d.B_max ? c.round_B : d.B_max;  // per-round buffers hold B_max
                B = (int)(left < (int64_t)cap ? left : (int64_t)cap);
            }
        }
        c.B = B;
        c.round_base = c.next_cand;
        c.S = c.S_raw = c.trunc = c.stop_at = 0;
        c.n_gray = 0;
        if (B > 0) c.epoch = (c.epoch + 1) & 0xFFFFFF;
        ntiles[u] = (B + kTile - 1) / kTile;
    }
    __syncthreads();
    // Tiles are handed out costliest universe first, so the long tiles start in
    // the first wave instead of trailing the round (order does not change results).
    for (int u = threadIdx.x; u < n; u += blockDim.x) {
        const int cu = ntiles[u] > 0 ? cost[u] : -1;
        int rank = 0;
        for (int v = 0; v < n; v++) {
            const int cv = ntiles[v] > 0 ? cost[v] : -1;
            rank += cv > cu || (cv == cu && v < u);
        }
        order[rank] = u;
    }
    __syncthreads();
    __shared__ int32_t wsum[8];
    int acc = 0;
    for (int b0 = 0; b0 < n; b0 += 256) {  // k_plan runs as one block of 256 threads
        const int i = b0 + threadIdx.x;
        const int nt = i < n ? ntiles[order[i]] : 0;
        int tot;
        const int p = block_excl_scan256(nt, wsum, &tot);
        if (i < n) {
            info->tile_off[i] = acc + p;
            info->tile_uni[i] = order[i];
        }
        acc += tot;
    }
    if (threadIdx.x == 0) {
        info->tile_off[n] = acc;
        info->total_tiles = acc;
        info->any_active = acc > 0;
        info->total_surv = 0;
        info->compact_done = 0;
        info->tile_next = 0;
        info->confl_next = 0;
        info->gemm_next = 0;
    }
}

// ------------------------------------------------------------- prefilter

// FP64 test of candidate idx against the committed packing.  Returns true
// when it is rejected.  Group mode: *g gets the single group touched (-1 none).
__device__ bool test64(const UniDev& d, int64_t n_slots, const double* alpha, const double* beta,
                       const double* a2, bool group, int32_t* g, int* nev, int* nvis = nullptr) {
    *g = -1;
    const int T = d.T, F1 = d.F + 1;
    if (d.dim == 1 && d.cross1d) {
        double P[kMaxF];
        for (int t = 0; t < T; t++) P[t] = eval64(d, alpha, beta, 1, a2[0], t);
        *nev = T;
        for (int64_t s = 0; s < n_slots; s++) {
            const Pt64* q = d.pts + UG_IDX(s * T + T - 1, d.slot_cap * T) + 1 - T;
            double d0 = torus_delta(P[0] - __ldcg(&q[0].c[0]));
            bool hit = hit1(d0, d.cell, d.inclusive);
            for (int t = 1; t < T && !hit; t++) {
                const double d1 = torus_delta(P[t] - __ldcg(&q[t].c[0]));
                hit = hit1(d1, d.cell, d.inclusive) || crosses_step(d0, d1);
                d0 = d1;
            }
            if (hit) {
                if (!group) return true;
                const int32_t gq = __ldcg(&q[0].gid);
                if (*g == -1)
                    *g = gq;
                else if (*g != gq)
                    return true;
            }
        }
        return false;
    }
    const int64_t cpt = cells_per_t(d);
    for (int oi = 0; oi < T; oi++) {
        const int t = __ldg(d.order + oi);
        double P[3];
        for (int ax = 0; ax < d.dim; ax++) P[ax] = eval64(d, alpha + ax * F1, beta + ax * F1, 1, a2[ax], t);
        *nev = oi + 1;
        if (contacts64(d, t, P, group, g, cpt, nvis)) return true;
    }
    return false;
}

// Diagnostic probe (braid_cuda3d.cu:1650-1660): n fresh candidates of the stream
// keyed by `seed` tested against the final packing (plain exclusion), counted per
// bin of the x axis's sin1 offset a2 over [-1, 1).
__global__ void __launch_bounds__(kTile) k_probe(const UniDev* __restrict__ U, int u, int64_t n_slots,
                                                 uint64_t seed, int64_t n, int bins,
                                                 unsigned long long* proposed, unsigned long long* accepted) {
    extern __shared__ unsigned long long probe_hist[];  // [2][bins]
    for (int i = threadIdx.x; i < 2 * bins; i += blockDim.x) probe_hist[i] = 0;
    __syncthreads();
    UniDev d = U[u];
    d.seed = seed;
    double alpha[3 * (kMaxF + 1)], beta[3 * (kMaxF + 1)], a2[3];
    int32_t bj[kMaxF];
    double wj[kMaxF];
    const int F1 = d.F + 1;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        if (d.rng == RNG_KNOT)
            gen_knot64(d, (uint64_t)i, alpha, beta, a2, bj, wj, 1);
        else
            for (int ax = 0; ax < d.dim; ax++) a2[ax] = gen_philox64(d, (uint64_t)i, ax, alpha + ax * F1, beta + ax * F1, 1);
        int32_t g;
        int nev;
        const bool free = !test64(d, n_slots, alpha, beta, a2, false, &g, &nev);
        int b = (int)floor((a2[0] + 1.0) * 0.5 * bins);
        b = b < 0 ? 0 : (b >= bins ? bins - 1 : b);
        atomicAdd(&probe_hist[b], 1ull);
        if (free) atomicAdd(&probe_hist[bins + b], 1ull);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < bins; i += blockDim.x) {
        if (probe_hist[i]) atomicAdd(&proposed[i], probe_hist[i]);
        if (probe_hist[bins + i]) atomicAdd(&accepted[i], probe_hist[bins + i]);
    }
}

__device__ __forceinline__ bool group_phase(const UniDev& d, const UniCtl& c) {
    return d.group_mode == GROUP_UNIQUE || (d.group_mode == GROUP_SUBPATH && c.phase == 2);
}

// --------------------------------------------------------------- compact


__global__ void __launch_bounds__(256) k_compact(const UniDev* __restrict__ U, UniCtl* ctl,
                                                 RoundInfo* info) {
    __shared__ int32_t wsum[8];
    __shared__ int32_t s_running;
    __shared__ bool s_last;
    const int u = blockIdx.x;
    const UniDev& d = U[u];
    UniCtl& c = ctl[u];
    const int B = c.B;
    const int nwords = (B + 31) >> 5;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_running = 0;
    __syncthreads();
    for (int base = 0; base < nwords; base += 256) {
        const int w = base + tid;
        uint32_t bits = w < nwords ? d.surv_bits[w] : 0u;
        if (w == nwords - 1 && (B & 31)) bits &= (1u << (B & 31)) - 1u;
        const int cnt = __popc(bits);
        int incl = cnt;
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        if (lane == 31) wsum[warp] = incl;
        __syncthreads();
        int wpre = 0, tot = 0;
        for (int k = 0; k < 8; k++) {
            if (k < warp) wpre += wsum[k];
            tot += wsum[k];
        }
        int rank = s_running + wpre + incl - cnt;
        while (bits) {
            const int bit = __ffs(bits) - 1;
            bits &= bits - 1;
            if (rank <= d.S_max) d.surv_off[UG_IDX(rank, d.S_max + 1)] = w * 32 + bit;
            rank++;
        }
        __syncthreads();
        if (tid == 0) s_running += tot;
        __syncthreads();
    }
    const int S_raw = s_running;
    const int S = S_raw < d.S_max ? S_raw : d.S_max;
    for (int r = tid; r < S; r += 256) d.ccount[r] = 0;
    if (tid == 0) {
        c.S_raw = S_raw;
        c.S = S;
        c.trunc = S;
        __threadfence();
        s_last = atomicAdd(&info->compact_done, 1) == info->n_uni - 1;
    }
    __syncthreads();
    if (s_last) {  // the last block: work offsets of every universe, as block scans
        __threadfence();
        const int n = info->n_uni;
        int acc = 0, sev = 0, spt = 0, acc_o = 0, sev_o = 0;
        for (int b0 = 0; b0 < n; b0 += 256) {
            const int v = b0 + tid;
            int Sv = 0, sevv = 0, sptv = 0, So = 0, sevo = 0;
            if (v < n) {
                Sv = *(volatile int32_t*)&ctl[v].S;
                sevv = ((Sv * U[v].dim + 31) >> 5) * ((U[v].T + 31) >> 5);
                sptv = Sv * U[v].T;
                // the same survivors and product tiles, universes in tile order (costliest first)
                const int uo = info->tile_uni[v];
                So = *(volatile int32_t*)&ctl[uo].S;
                sevo = ((So * U[uo].dim + 31) >> 5) * ((U[uo].T + 31) >> 5);
            }
            int t1, t2, t3, t4, t5;
            const int p1 = block_excl_scan256(Sv, wsum, &t1);
            const int p2 = block_excl_scan256(sevv, wsum, &t2);
            const int p3 = block_excl_scan256(sptv, wsum, &t3);
            const int p4 = block_excl_scan256(So, wsum, &t4);
            const int p5 = block_excl_scan256(sevo, wsum, &t5);
            if (v < n) {
                info->surv_off[v] = acc + p1;
                info->sev_off[v] = sev + p2;
                info->spt_off[v] = spt + p3;
                info->surv_off_o[v] = acc_o + p4;
                info->sev_off_o[v] = sev_o + p5;
            }
            acc += t1;
            sev += t2;
            spt += t3;
            acc_o += t4;
            sev_o += t5;
        }
        if (tid == 0) {
            info->surv_off[n] = acc;
            info->sev_off[n] = sev;
            info->spt_off[n] = spt;
            info->surv_off_o[n] = acc_o;
            info->sev_off_o[n] = sev_o;
            info->total_surv = acc;
            info->total_sev = sev;
            info->total_spt = spt;
        }
    }
}

// ------------------------------------------------------------ survivors

// Round table entry of (timestep t, block lin): one 8-byte word per (t, block),
// epoch in the high half so no table is ever cleared.  A direct table replaced an
// open-addressing hash keyed by (epoch, t, block): one exchange per insert instead of
// a probe, a compare-and-swap and an exchange, and a quarter of the memory.
__device__ __forceinline__ uint64_t* rentry(const UniDev& d, int t, int64_t lin) {
    return d.rhead + UG_IDX((int64_t)t * d.rblocks + lin, (int64_t)d.T * d.rblocks);
}
// Head survivor of the chain of (t, block) this round (-1 none).
__device__ __forceinline__ int32_t rtab_head(const UniDev& d, int epoch, int t, int64_t lin) {
    const uint64_t v = __ldcg(rentry(d, t, lin));
    return (v >> 32) == (uint64_t)(uint32_t)epoch ? (int32_t)(uint32_t)v : -1;
}

// Warp-cooperative FP64 regeneration of axis ax of candidate idx (Philox
// stream) into shared memory: Philox blocks are spread over the lanes, the
// normalisation sum runs in ascending b on lane 0 -- the same operations, in
// the same order, as the thread-per-candidate gen_philox64, so the
// coefficients are identical.
__device__ __forceinline__ void warp_gen64_axis(const UniDev& d, uint64_t idx, int ax, double* alpha, double* beta,
                                                double* a2, int lane) {
    const int F = d.F, F1 = F + 1;
    double* al = alpha + ax * F1;
    double* bt = beta + ax * F1;
    for (int p = lane; 2 * p <= F; p += 32) {
        const uint4 o = philox_block(d.seed, idx, ax, p);
        if (p == 0) {
            a2[ax] = d.pin ? 0.0 : (double)o.x * (1.0 / 2147483648.0) - 1.0;
            continue;
        }
        const int be = 2 * p, bo = 2 * p + 1;
        const double Ee = -log(((double)o.x + 0.5) * (1.0 / 4294967296.0));
        al[be] = (o.z & 1u) ? -Ee : Ee;
        bt[be] = (double)(o.z >> 1) * (1.0 / 2147483648.0) * kPi;
        if (bo <= F) {
            const double Eo = -log(((double)o.y + 0.5) * (1.0 / 4294967296.0));
            al[bo] = (o.w & 1u) ? -Eo : Eo;
        }
    }
    __syncwarp();
    double sum = 0.0;
    if (lane == 0)
        for (int b = 2; b <= F; b++) sum += fabs(al[b]);
    sum = __shfl_sync(0xffffffffu, sum, 0);
    for (int b = 2 + lane; b <= F; b += 32) {
        const double e = al[b];
        double amp = fabs(e) / sum / (double)b;
        if (e < 0.0) amp = -amp;
        if (b & 1) {
            al[b] = amp;
            bt[b] = 0.0;
        } else {
            double sf, cf;
            sincos(bt[b], &sf, &cf);
            al[b] = amp * cf;
            bt[b] = amp * sf;
        }
    }
    __syncwarp();
}

// All axes of candidate idx by one warp (the knot stream is sequential: lane 0
// replays it).
__device__ __forceinline__ void warp_gen64(const UniDev& d, uint64_t idx, double* alpha, double* beta,
                                       double* a2, int32_t* bj, double* wj, int lane) {
    if (d.rng == RNG_KNOT) {
        if (lane == 0) gen_knot64(d, idx, alpha, beta, a2, bj, wj, 1);
        __syncwarp();
    } else {
        for (int ax = 0; ax < d.dim; ax++) warp_gen64_axis(d, idx, ax, alpha, beta, a2, lane);
    }
}

// Rows r * dim + ax of the term-ordered coefficient matrix of one survivor.
__device__ __forceinline__ void store_coef_rows(const UniDev& d, int r, const double* alpha, const double* beta,
                                                const double* a2, int lane) {
    const int F = d.F, F1 = F + 1, R = d.Rpad;
    [[maybe_unused]] const int64_t ncoef = (int64_t)d.K * R;
    for (int ax = 0; ax < d.dim; ax++) {
        const int row = r * d.dim + ax;
        const double* al = alpha + ax * F1;
        const double* bt = beta + ax * F1;
        for (int b = 2 + lane; b <= F; b += 32) {
            const int64_t k = kseq_s(b);
            d.coef[UG_IDX(k * R + row, ncoef)] = al[b];
            if (!(b & 1)) d.coef[UG_IDX((k + 1) * R + row, ncoef)] = bt[b];
        }
        if (lane == 0) d.a2row[UG_IDX(row, R)] = a2[ax];
    }
}

// Survivor trajectories in three steps.
//
// k_surv_gen: one warp per survivor regenerates its FP64 coefficients
// (warp-parallel Philox blocks, sequential normalisation sum in ascending b --
// the same operations as the thread-per-candidate prefilter, so identical
// values) and stores them as rows r * dim + ax of the term-ordered matrix coef.
__global__ void __launch_bounds__(32 * kSurvWarps) k_surv_gen(const UniDev* __restrict__ U,
                                                                UniCtl* ctl, RoundInfo* info, int warp_bytes) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    unsigned char* my = smem_raw + (size_t)wib * warp_bytes;
    double* alpha = (double*)my;
    double* beta = alpha + 3 * (kMaxF + 1);
    double* a2 = beta + 3 * (kMaxF + 1);
    double* wj = a2 + 3;
    int32_t* bj = (int32_t*)(wj + kMaxF);
    const int n_uni = info->n_uni, total = info->total_surv;
    const int gwarp = blockIdx.x * kSurvWarps + wib, nwarps = gridDim.x * kSurvWarps;
    for (int item = gwarp; item < total; item += nwarps) {
        const int u = find_uni(info->surv_off, n_uni, item);
        const int r = item - info->surv_off[u];
        const UniDev& d = U[u];
        const UniCtl& c = ctl[u];
        const uint64_t idx = (uint64_t)(c.round_base + d.surv_off[UG_IDX(r, d.S_max + 1)]);
        if (d.rng == RNG_PHILOX) {
            // one axis at a time in a (F+1)-entry buffer pair, rows written as they are
            // finished: warp_gen64's operations per axis, a quarter of its shared memory
            const int F = d.F, R = d.Rpad;
            [[maybe_unused]] const int64_t ncoef = (int64_t)d.K * R;
            double* al = (double*)my;
            double* bt = al + (kMaxF + 1);
            for (int ax = 0; ax < d.dim; ax++) {
                const int row = r * d.dim + ax;
                for (int p = lane; 2 * p <= F; p += 32) {
                    const uint4 o = philox_block(d.seed, idx, ax, p);
                    if (p == 0) {
                        d.a2row[UG_IDX(row, R)] = d.pin ? 0.0 : (double)o.x * (1.0 / 2147483648.0) - 1.0;
                        continue;
                    }
                    const int be = 2 * p, bo = 2 * p + 1;
                    const double Ee = -log(((double)o.x + 0.5) * (1.0 / 4294967296.0));
                    al[be] = (o.z & 1u) ? -Ee : Ee;
                    bt[be] = (double)(o.z >> 1) * (1.0 / 2147483648.0) * kPi;
                    if (bo <= F) {
                        const double Eo = -log(((double)o.y + 0.5) * (1.0 / 4294967296.0));
                        al[bo] = (o.w & 1u) ? -Eo : Eo;
                    }
                }
                __syncwarp();
                double sum = 0.0;
                if (lane == 0)
                    for (int b = 2; b <= F; b++) sum += fabs(al[b]);
                sum = __shfl_sync(0xffffffffu, sum, 0);
                for (int b = 2 + lane; b <= F; b += 32) {
                    const double e = al[b];
                    double amp = fabs(e) / sum / (double)b;
                    if (e < 0.0) amp = -amp;
                    const int64_t k = kseq_s(b);
                    if (b & 1) {
                        d.coef[UG_IDX(k * R + row, ncoef)] = amp;
                    } else {
                        double sf, cf;
                        sincos(bt[b], &sf, &cf);
                        d.coef[UG_IDX(k * R + row, ncoef)] = amp * cf;
                        d.coef[UG_IDX((k + 1) * R + row, ncoef)] = amp * sf;
                    }
                }
                __syncwarp();
            }
            continue;
        }
        warp_gen64(d, idx, alpha, beta, a2, bj, wj, lane);
        store_coef_rows(d, r, alpha, beta, a2, lane);
        __syncwarp();
    }
}

// Checkpoint restore: the coefficient rows of m given admissions (explicit
// candidate indices) of universe u, as k_surv_gen writes them for survivors.
__global__ void __launch_bounds__(32 * kSurvWarps) k_restore_gen(const UniDev* __restrict__ U, int u,
                                                                   const int64_t* __restrict__ idx, int m) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    unsigned char* my = smem_raw + (size_t)wib * kSurvSmemPerWarp;
    double* alpha = (double*)my;
    double* beta = alpha + 3 * (kMaxF + 1);
    double* a2 = beta + 3 * (kMaxF + 1);
    double* wj = a2 + 3;
    int32_t* bj = (int32_t*)(wj + kMaxF);
    const UniDev& d = U[u];
    const int gwarp = blockIdx.x * kSurvWarps + wib, nwarps = gridDim.x * kSurvWarps;
    for (int r = gwarp; r < m; r += nwarps) {
        warp_gen64(d, (uint64_t)idx[r], alpha, beta, a2, bj, wj, lane);
        store_coef_rows(d, r, alpha, beta, a2, lane);
        __syncwarp();
    }
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(smem)),
                 "l"(gmem)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// k_surv_gemm: X[row][t] = wrap(a2 + invsinz_t * sum_k coef[k][row] KT[k][t]),
// one warp per 32-row x 32-timestep tile.  Lane (rg, tg) owns rows
// row0 + 0..3 and timesteps t0 + 8 jj + {0,1}; every (row, t) is a single FMA
// chain in ascending k, i.e. eval64's operations in eval64's order.  Each warp
// streams its tile's A rows and B columns through shared memory in chunks of
// kGemmKC terms, two stages deep (cp.async), so the next chunk is in flight while
// the current one is multiplied.
__global__ void __launch_bounds__(128) k_surv_gemm(const UniDev* __restrict__ U, UniCtl* ctl,
                                                   RoundInfo* info) {
    extern __shared__ __align__(16) double gemm_smem[];  // [warp][stage][A | B][kGemmKC][32]
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    double* wsm = gemm_smem + (size_t)wib * (2 * 2 * kGemmKC * 32);
    const int n_uni = info->n_uni, total = info->total_sev;
    const int rg = lane >> 2, tg = lane & 3;
    // tiles handed out one at a time, costliest universes first (a tile's cost is
    // its universe's term count K, 24 to 384); the next claimed when one starts
    int item = 0, next = 0;
    if (lane == 0) item = atomicAdd(&info->gemm_next, 1);
    item = __shfl_sync(0xffffffffu, item, 0);
    for (; item < total; item = __shfl_sync(0xffffffffu, next, 0)) {
        if (lane == 0) next = atomicAdd(&info->gemm_next, 1);
        const int pos = find_uni(info->sev_off_o, n_uni, item);
        const int u = info->tile_uni[pos];
        const int local = item - info->sev_off_o[pos];
        const UniDev& d = U[u];
        const int T = d.T, dim = d.dim, K = d.K, R = d.Rpad, TP = d.Tpad;
        const int ntb = (T + 31) >> 5;
        const int rb = local / ntb, tb = local - rb * ntb;
        const int row0 = rb * 32 + rg * 4;
        const int t0 = tb * 32 + 2 * tg;
        const double* Ag = d.coef + rb * 32;  // tile rows [rb*32, rb*32+32) < Rpad
        const double* Bg = d.KT + tb * 32;    // tile timesteps [tb*32, tb*32+32) < Tpad
        // chunk ch: terms [ch*KC, min(K, ch*KC+KC)), 16-byte pieces (16 per 32-double row)
        auto issue = [&](int stage, int k0) {
            double* As = wsm + stage * (2 * kGemmKC * 32);
            double* Bs = As + kGemmKC * 32;
            for (int i = lane; i < kGemmKC * 16; i += 32) {
                const int kk = i >> 4, pc = (i & 15) * 2;
                if (k0 + kk < K) {
                    cp_async16(As + kk * 32 + pc, Ag + (size_t)(k0 + kk) * R + pc);
                    cp_async16(Bs + kk * 32 + pc, Bg + (size_t)(k0 + kk) * TP + pc);
                }
            }
            cp_async_commit();
        };
        double acc[4][8];
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 8; j++) acc[i][j] = 0.0;
        const int nch = (K + kGemmKC - 1) / kGemmKC;
        issue(0, 0);
        for (int ch = 0; ch < nch; ch++) {
            if (ch + 1 < nch) {
                issue((ch + 1) & 1, (ch + 1) * kGemmKC);
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
            __syncwarp();
            const double* As = wsm + (ch & 1) * (2 * kGemmKC * 32) + rg * 4;
            const double* Bs = wsm + (ch & 1) * (2 * kGemmKC * 32) + kGemmKC * 32 + 2 * tg;
            const int kn = min(kGemmKC, K - ch * kGemmKC);
#pragma unroll 4
            for (int kk = 0; kk < kn; kk++) {
                const double2 a01 = *(const double2*)(As + kk * 32);
                const double2 a23 = *(const double2*)(As + kk * 32 + 2);
                const double av[4] = {a01.x, a01.y, a23.x, a23.y};
                double bv[8];
#pragma unroll
                for (int jj = 0; jj < 4; jj++) {
                    const double2 b2 = *(const double2*)(Bs + kk * 32 + 8 * jj);
                    bv[2 * jj] = b2.x;
                    bv[2 * jj + 1] = b2.y;
                }
#pragma unroll
                for (int i = 0; i < 4; i++)
#pragma unroll
                    for (int j = 0; j < 8; j++) acc[i][j] = fma(av[i], bv[j], acc[i][j]);
            }
            __syncwarp();  // the stage is refilled by the issue of chunk ch + 2
        }
        const int nrows = ctl[u].S * dim;
        [[maybe_unused]] const int64_t nspos = (int64_t)d.S_max * T;
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int row = row0 + i;
            if (row >= nrows) continue;
            const int r = row / dim, ax = row - r * dim;
            const double a2 = d.a2row[UG_IDX(row, R)];
#pragma unroll
            for (int j = 0; j < 8; j++) {
                const int t = t0 + 8 * (j >> 1) + (j & 1);
                if (t < T)
                    d.spos[UG_IDX((int64_t)r * T + t, nspos)].c[ax] =
                        torus_wrap(fma(acc[i][j], __ldg(d.invsinz + t), a2));
            }
        }
    }
}

// Round-table block of a cell: 2^rblock_shift cells per axis (host-chosen per
// universe, at least 2), so the 3 neighbour cells of a point span at most 2
// blocks per axis (3 only at the seam of a partial last block).
static_assert(2 * kMaxF <= 1024, "k_conflicts packs block coordinates in 10 bits");
__device__ __forceinline__ int rblock_gw(const UniDev& d) {
    return (d.gw + (1 << d.rblock_shift) - 1) >> d.rblock_shift;
}

// k_surv_hash: one thread per survivor timestep inserts the point into the
// round table (entry: t, block; tagged with the epoch).
__global__ void __launch_bounds__(256) k_surv_hash(const UniDev* __restrict__ U, UniCtl* ctl,
                                                   RoundInfo* info) {
    const int n_uni = info->n_uni, total = info->total_spt;
    for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < total; w += gridDim.x * blockDim.x) {
        const int u = find_uni(info->spt_off, n_uni, w);
        const UniDev& d = U[u];
        const UniCtl& c = ctl[u];
        const int T = d.T;
        const int local = w - info->spt_off[u];
        const int r = local / T, t = local - r * T;
        Pt64* q = d.spos + UG_IDX((int64_t)r * T + t, (int64_t)d.S_max * T);
        int bc[3] = {0, 0, 0};
#pragma unroll
        for (int ax = 0; ax < 3; ax++) {
            if (ax < d.dim)
                bc[ax] = cell_of(q->c[ax], d.cell, d.gw) >> d.rblock_shift;
            else
                q->c[ax] = 0.0;
        }
        const uint64_t ep = (uint64_t)(uint32_t)c.epoch;
        const uint64_t old = atomicExch((unsigned long long*)rentry(d, t, lin_cell(bc, d.dim, rblock_gw(d))),
                                        (unsigned long long)((ep << 32) | (uint32_t)r));
        q->next = (old >> 32) == ep ? (int32_t)(uint32_t)old : -1;
        q->gid = -1;
    }
}

// Candidates the mixed prefilter could not decide (guard band, or universes
// outside the tensor-core path), in index order, per universe.
__global__ void __launch_bounds__(256) k_gray_compact(const UniDev* __restrict__ U, UniCtl* ctl,
                                                      RoundInfo* info, int all) {
    __shared__ int32_t wsum[8];
    __shared__ int32_t s_running;
    __shared__ bool s_last;
    const int u = blockIdx.x;
    const UniDev& d = U[u];
    UniCtl& c = ctl[u];
    const int B = c.B;
    const int nwords = (B + 31) >> 5;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_running = 0;
    __syncthreads();
    for (int base = 0; base < nwords; base += 256) {
        const int w = base + tid;
        // all: the FP64 form, every candidate of the round goes to the warp test
        uint32_t bits = w < nwords ? (all ? 0xffffffffu : d.gray_bits[w]) : 0u;
        if (all && w < nwords) d.surv_bits[UG_IDX(w, d.B_max / 32)] = 0u;
        if (w == nwords - 1 && (B & 31)) bits &= (1u << (B & 31)) - 1u;
        const int cnt = __popc(bits);
        int incl = cnt;
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        if (lane == 31) wsum[warp] = incl;
        __syncthreads();
        int wpre = 0, tot = 0;
        for (int k = 0; k < 8; k++) {
            if (k < warp) wpre += wsum[k];
            tot += wsum[k];
        }
        int rank = s_running + wpre + incl - cnt;
        while (bits) {
            const int bit = __ffs(bits) - 1;
            bits &= bits - 1;
            d.gray_off[UG_IDX(rank, d.B_max)] = w * 32 + bit;
            rank++;
        }
        __syncthreads();
        if (tid == 0) s_running += tot;
        __syncthreads();
    }
    if (tid == 0) {
        c.n_gray = s_running;
        __threadfence();
        s_last = atomicAdd(&info->gray_done, 1) == info->n_uni - 1;
    }
    __syncthreads();
    if (s_last) {  // the last block: offsets of every universe's undecided candidates
        __threadfence();
        const int n = info->n_uni;
        int acc = 0;
        for (int b0 = 0; b0 < n; b0 += 256) {
            const int v = b0 + tid;
            const int g = v < n ? *(volatile int32_t*)&ctl[v].n_gray : 0;
            int tot;
            const int p = block_excl_scan256(g, wsum, &tot);
            if (v < n) info->gray_pref[v] = acc + p;
            acc += tot;
        }
        if (tid == 0) {
            info->gray_pref[n] = acc;
            info->total_gray = acc;
            info->gray_done = 0;
        }
    }
}

// FP64 test of one candidate per group of WPI warps: FP64 regeneration and the
// exact test against the committed packing, timesteps (1+1D: paths) spread
// over the group's lanes.  WPI = 1 serves the FP64 form (every candidate of the
// round: many items, throughput); WPI = kSurvWarps the guard-band retest of the
// mixed form (few items per round, each of which would otherwise bound the
// launch by one warp's latency): the axes are generated by separate warps and
// four times the lanes share the timesteps.
template <int WPI>
__device__ __forceinline__ void group_sync() {
    if (WPI == 1)
        __syncwarp();
    else
        __syncthreads();
}

// (a register cap instead of launch bounds: with launch bounds alone ptxas keeps
// the WPI = 1 form at 64 registers and spills)
template <int WPI>
__global__ void __maxnreg__(128) k_confirm64w(const UniDev* __restrict__ U,
                                                                  UniCtl* ctl, RoundInfo* info, int all) {
    static_assert(WPI == 1 || WPI == kSurvWarps, "a group is one warp or the whole block");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int kG = kSurvWarps / WPI;  // groups per block
    constexpr int kGT = 32 * WPI;         // threads per group
    __shared__ int32_t s_hit[kG];
    __shared__ int32_t s_first[kSurvWarps], s_rej[kSurvWarps];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int grp = wib / WPI, wig = wib % WPI, gt = wig * 32 + lane;
    unsigned char* my = smem_raw + (size_t)grp * kConfSmemPerWarp;
    double* alpha = (double*)my;
    double* beta = alpha + 3 * (kMaxF + 1);
    double* a2 = beta + 3 * (kMaxF + 1);
    double* wj = a2 + 3;
    int32_t* bj = (int32_t*)(wj + kMaxF);
    double* P1 = (double*)(my + kSurvSmemPerWarpBase);
    volatile int32_t* vhit = &s_hit[grp];
    const int n_uni = info->n_uni, total = info->total_gray;
    const int ggrp = blockIdx.x * kG + grp, ngrp = gridDim.x * kG;
    for (int item = ggrp; item < total; item += ngrp) {
        const int u = find_uni(info->gray_pref, n_uni, item);
        const UniDev& d = U[u];
        UniCtl& c = ctl[u];
        const int off = d.gray_off[UG_IDX(item - info->gray_pref[u], d.B_max)];
        const uint64_t idx = (uint64_t)(c.round_base + off);
        const int T = d.T;
        if (d.rng == RNG_KNOT || WPI == 1) {
            if (wig == 0) warp_gen64(d, idx, alpha, beta, a2, bj, wj, lane);
        } else if (wig < d.dim) {
            warp_gen64_axis(d, idx, wig, alpha, beta, a2, lane);
        }
        if (gt == 0) *vhit = 0;
        group_sync<WPI>();
        const bool group = group_phase(d, c);
        int32_t g = -1;
        bool hitl = false;
        int nev = 0, nvis = 0;
        if (d.dim == 1 && d.cross1d) {
            for (int t = gt; t < T; t += kGT) P1[t] = eval64(d, alpha, beta, 1, a2[0], t);
            group_sync<WPI>();
            nev = gt == 0 ? T : 0;
            for (int64_t s = gt; s < c.n_slots && !(hitl && !group); s += kGT) {
                if (!group && *vhit) break;  // another lane of the group found a contact
                const Pt64* q = d.pts + UG_IDX(s * T + T - 1, d.slot_cap * T) + 1 - T;
                double d0 = torus_delta(P1[0] - __ldcg(&q[0].c[0]));
                bool hit = hit1(d0, d.cell, d.inclusive);
                // the path's points 4 timesteps at a time (4 independent loads in flight)
                for (int t0 = 1; t0 < T && !hit; t0 += 4) {
                    double qv[4];
#pragma unroll
                    for (int k = 0; k < 4; k++) qv[k] = t0 + k < T ? __ldcg(&q[t0 + k].c[0]) : 0.0;
#pragma unroll
                    for (int k = 0; k < 4; k++) {
                        if (hit || t0 + k >= T) break;
                        const double d1 = torus_delta(P1[t0 + k] - qv[k]);
                        hit = hit1(d1, d.cell, d.inclusive) || crosses_step(d0, d1);
                        d0 = d1;
                    }
                }
                if (hit) {
                    if (!group) {
                        hitl = true;
                        *vhit = 1;
                    } else {
                        const int32_t gq = __ldcg(&q[0].gid);
                        if (g == -1)
                            g = gq;
                        else if (g != gq)
                            hitl = true;
                    }
                }
            }
        } else {
            const int64_t cpt = cells_per_t(d);
            for (int oi0 = 0; oi0 < T; oi0 += kGT) {
                const int oi = oi0 + gt;
                if (oi < T && !hitl) {
                    const int t = __ldg(d.order + oi);
                    double P[3];
                    if (d.dim == 3)
                        eval64x<3>(d, alpha, beta, a2, t, P);
                    else if (d.dim == 2)
                        eval64x<2>(d, alpha, beta, a2, t, P);
                    else
                        eval64x<1>(d, alpha, beta, a2, t, P);
                    nev++;
                    hitl = contacts64(d, t, P, group, &g, cpt, all ? &nvis : nullptr);
                }
                if (__any_sync(0xffffffffu, hitl)) {
                    if (lane == 0) *vhit = 1;
                    break;
                }
                if (WPI > 1 && *vhit) break;
            }
        }
        // merge the lanes of each warp, then the warps of the group: any rejection,
        // or (group rounds) two distinct groups touched
        bool rej = __any_sync(0xffffffffu, hitl);
        int32_t first = -1;
        for (int o = 0; o < 32; o++) {
            const int32_t v = __shfl_sync(0xffffffffu, g, o);
            if (first == -1) first = v;
        }
        if (group) rej = rej || __any_sync(0xffffffffu, g != -1 && g != first);
        for (int o = 16; o > 0; o >>= 1) nev += __shfl_xor_sync(0xffffffffu, nev, o);
        for (int o = 16; o > 0; o >>= 1) nvis += __shfl_xor_sync(0xffffffffu, nvis, o);
        if (lane == 0) {
            if (nev) atomicAdd((unsigned long long*)&c.evals_fp64, (unsigned long long)nev);
            if (all && nev) atomicAdd((unsigned long long*)&c.evals, (unsigned long long)nev);
            if (nvis) atomicAdd((unsigned long long*)&c.visits, (unsigned long long)nvis);
        }
        if (WPI > 1) {
            if (lane == 0) {
                s_first[wib] = first;
                s_rej[wib] = rej ? 1 : 0;
            }
            __syncthreads();
            first = -1;
            rej = false;
            for (int w = 0; w < WPI; w++) {
                const int32_t v = s_first[grp * WPI + w];
                rej = rej || s_rej[grp * WPI + w] != 0 || (v != -1 && first != -1 && v != first);
                if (first == -1) first = v;
            }
        }
        if (gt == 0) {
            if (!rej) atomicOr(&d.surv_bits[UG_IDX(off >> 5, d.B_max / 32)], 1u << (off & 31));
            if (d.group_mode != GROUP_NONE) d.g0[UG_IDX(off, d.B_max)] = first;
        }
        group_sync<WPI>();
    }
}

cudaError_t confirm64w_set_smem() {
    cudaError_t e = cudaFuncSetAttribute(k_confirm64w<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)(kSurvWarps * kConfSmemPerWarp));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_confirm64w<kSurvWarps>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kConfSmemPerWarp);
    return e;
}

void launch_confirm64w(int all, int nsm, const UniDev* U, UniCtl* ctl, RoundInfo* info, cudaStream_t st) {
    if (all)
        k_confirm64w<1><<<nsm * 4, 32 * kSurvWarps, kSurvWarps * kConfSmemPerWarp, st>>>(U, ctl, info, 1);
    else
        k_confirm64w<kSurvWarps><<<nsm * 4, 32 * kSurvWarps, kConfSmemPerWarp, st>>>(U, ctl, info, 0);
}

// One warp per survivor r: the set of earlier survivors r' < r that it
// touches (Chebyshev contact at any timestep; plus crossings in 1+1D).
__global__ void __launch_bounds__(128) k_conflicts(const UniDev* __restrict__ U, UniCtl* ctl,
                                                    RoundInfo* info) {
    __shared__ int32_t s_cnt[4];
    __shared__ int32_t s_list[4][kConflictCap];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int n_uni = info->n_uni, total = info->total_surv;
    volatile int32_t* cnt = &s_cnt[wib];
    volatile int32_t* lst = s_list[wib];
    // Survivors are handed out one at a time, costliest universes first (their cost
    // differs by the timesteps and dimension); the next one is claimed when an item
    // starts so the atomic's latency hides behind the item.
    int item = 0;
    if (lane == 0) item = atomicAdd(&info->confl_next, 1);
    item = __shfl_sync(0xffffffffu, item, 0);
    while (item < total) {
        int next = 0;
        if (lane == 0) next = atomicAdd(&info->confl_next, 1);
        const int pos = find_uni(info->surv_off_o, n_uni, item);
        const int u = info->tile_uni[pos];
        const int r = item - info->surv_off_o[pos];
        const UniDev& d = U[u];
        UniCtl& c = ctl[u];
        const int T = d.T;
        if (lane == 0) *cnt = 0;
        __syncwarp();
        auto add = [&](int32_t r2) {
            const int n = *cnt < kConflictCap ? *cnt : kConflictCap;
            for (int i = 0; i < n; i++)
                if (lst[i] == r2) return;
            const int pos = atomicAdd((int32_t*)cnt, 1);
            if (pos < kConflictCap) lst[pos] = r2;
        };
        if (d.dim == 1 && d.cross1d) {
            const Pt64* P = d.spos + UG_IDX((int64_t)r * T + T - 1, (int64_t)d.S_max * T) + 1 - T;
            for (int r2 = lane; r2 < r; r2 += 32) {
                const Pt64* Q = d.spos + UG_IDX((int64_t)r2 * T + T - 1, (int64_t)d.S_max * T) + 1 - T;
                double d0 = torus_delta(P[0].c[0] - Q[0].c[0]);
                bool hit = hit1(d0, d.cell, d.inclusive);
                // both paths' points 4 timesteps at a time (independent loads in flight)
                for (int t0 = 1; t0 < T && !hit; t0 += 4) {
                    double pv[4], qv[4];
#pragma unroll
                    for (int k = 0; k < 4; k++) {
                        pv[k] = t0 + k < T ? P[t0 + k].c[0] : 0.0;
                        qv[k] = t0 + k < T ? Q[t0 + k].c[0] : 0.0;
                    }
#pragma unroll
                    for (int k = 0; k < 4; k++) {
                        if (hit || t0 + k >= T) break;
                        const double d1 = torus_delta(pv[k] - qv[k]);
                        hit = hit1(d1, d.cell, d.inclusive) || crosses_step(d0, d1);
                        d0 = d1;
                    }
                }
                if (hit) add(r2);
            }
        } else {
            const int gw = d.gw, gwb = rblock_gw(d), rbs = d.rblock_shift;
            for (int t = lane; t < T; t += 32) {
                const Pt64 P = d.spos[UG_IDX((int64_t)r * T + t, (int64_t)d.S_max * T)];
                // distinct round-table blocks of the 3 neighbour cells per axis:
                // bl[ax] packs up to three 10-bit block coordinates, nbk[ax] counts them
                // (registers only: every index below is a compile-time constant)
                uint32_t bl[3] = {0u, 0u, 0u};
                int nbk[3] = {1, 1, 1};
#pragma unroll
                for (int ax = 0; ax < 3; ax++) {
                    if (ax < d.dim) {
                        const int c0 = cell_of(P.c[ax], d.cell, gw);
                        const uint32_t v0 = (uint32_t)((c0 == 0 ? gw - 1 : c0 - 1) >> rbs);
                        const uint32_t v1 = (uint32_t)(c0 >> rbs);
                        const uint32_t v2 = (uint32_t)((c0 == gw - 1 ? 0 : c0 + 1) >> rbs);
                        uint32_t pk = v0;
                        int n = 1;
                        if (v1 != v0) pk |= v1 << (10 * n++);
                        if (v2 != v0 && v2 != v1) pk |= v2 << (10 * n++);
                        bl[ax] = pk;
                        nbk[ax] = n;
                    }
                }
                for (int i0 = 0; i0 < nbk[0]; i0++)
                    for (int i1 = 0; i1 < nbk[1]; i1++)
                        for (int i2 = 0; i2 < nbk[2]; i2++) {
                            const int bc[3] = {(int)((bl[0] >> (10 * i0)) & 1023u),
                                               (int)((bl[1] >> (10 * i1)) & 1023u),
                                               (int)((bl[2] >> (10 * i2)) & 1023u)};
                            int32_t r2 = rtab_head(d, c.epoch, t, lin_cell(bc, d.dim, gwb));
                            while (r2 >= 0) {
                                if (r2 == r) {  // this survivor's own point: its link is in P
                                    r2 = P.next;
                                    continue;
                                }
                                const Pt64* Q = d.spos + UG_IDX((int64_t)r2 * T + t, (int64_t)d.S_max * T);
                                if (r2 < r && pair_hit64(d, P.c, Q->c)) add(r2);
                                r2 = Q->next;
                            }
                        }
            }
        }
        __syncwarp();
        // more than kConflictCap contacts: the list keeps kConflictCap of them and the
        // count says so; the resolver rejects on any admitted one and otherwise stops
        // the round at this survivor
        const int n = *cnt;
        const int ns = n < kConflictCap ? n : kConflictCap;
        for (int i = lane; i < ns; i += 32) d.clist[UG_IDX((int64_t)r * kConflictCap + i, (int64_t)d.S_max * kConflictCap)] = lst[i];
        if (lane == 0) d.ccount[UG_IDX(r, d.S_max)] = n;
        __syncwarp();
        item = __shfl_sync(0xffffffffu, next, 0);
    }
}

// ------------------------------------------------------------- resolver

// One warp per universe: survivors in index order; admit survivor r iff the
// sequential-RSA rule holds against the round's earlier admissions.
__global__ void __launch_bounds__(32) k_greedy(const UniDev* __restrict__ U, UniCtl* ctl,
                                               RoundInfo* info) {
    extern __shared__ int32_t greedy_smem[];
    int32_t* acc_s = greedy_smem;
    int32_t* gid_s = greedy_smem + kSmaxCap;
    const int u = blockIdx.x;
    const int lane = threadIdx.x;
    const UniDev& d = U[u];
    UniCtl& c = ctl[u];
    if (c.B == 0) return;
    const int S = c.S;
    const int S_eff = c.trunc < S ? c.trunc : S;
    const bool group = group_phase(d, c);
    const bool unique_group = d.group_mode == GROUP_UNIQUE;
    const int64_t room = d.slot_cap - c.n_slots;
    int k = 0, stop_at = S_eff;
    int64_t n_unique = c.n_unique, n_sub = c.n_sub;
    bool grow = false, hit_max = false, undecided = false;
    // Plain rounds: 32 survivors per step.  Each lane gathers its survivor's
    // listed contacts -- admitted ones from earlier steps (certain rejection)
    // and a bit mask of the earlier lanes of this step -- and the warp then
    // decides the 32 in index order from those masks: the same decisions as the
    // one-at-a-time loop below, which group rounds use.
    for (int r0 = 0; !group && r0 < S_eff; r0 += 32) {
        const int r = r0 + lane, nvalid = min(32, S_eff - r0);
        uint32_t dep = 0;
        bool ext = false, over = false;
        if (lane < nvalid) {
            const int n_all = d.ccount[UG_IDX(r, d.S_max)];
            over = n_all > kConflictCap;
            const int n = over ? kConflictCap : n_all;
            const int32_t* lst = d.clist + UG_IDX((int64_t)r * kConflictCap, (int64_t)d.S_max * kConflictCap);
            for (int i = 0; i < n; i++) {
                const int r2 = lst[i];
                if (r2 < r0)
                    ext |= acc_s[UG_IDX(r2, kSmaxCap)] >= 0;
                else
                    dep |= 1u << (r2 - r0);
            }
        }
        // In-order greedy over the step's lanes: a lane decides once every lane it
        // depends on has decided (dependencies point to lower lanes only, so the
        // lowest undecided lane is always ready; one pass per link of the longest
        // dependency chain, usually one).
        const uint32_t valid = nvalid >= 32 ? 0xffffffffu : ((1u << nvalid) - 1u);
        uint32_t und = valid, accm = 0;
        while (und) {
            const bool ready = ((und >> lane) & 1u) && !(dep & und);
            accm |= __ballot_sync(0xffffffffu, ready && !ext && !(dep & accm));
            und &= ~__ballot_sync(0xffffffffu, ready);
        }
        // Where the one-at-a-time scan would stop: at lane j it first checks the
        // room left (stop before j), then an admitted j with an over-full list
        // (undecided: stop before j), then the unique cap (stop after j).
        const int acc_before = __popc(accm & ((1u << lane) - 1u));
        const bool mine = (accm >> lane) & 1u;
        const uint32_t b_room = __ballot_sync(0xffffffffu, lane < nvalid && k + acc_before >= room);
        const uint32_t b_over = __ballot_sync(0xffffffffu, mine && over);
        const uint32_t b_max = __ballot_sync(
            0xffffffffu, mine && c.phase == 1 && c.max_n > 0 && n_unique + acc_before + 1 >= c.max_n);
        int stop = -1;
        if (b_room | b_over | b_max) {
            const int j = __ffs(b_room | b_over | b_max) - 1;
            if ((b_room >> j) & 1u) {
                stop = j;
                grow = true;
            } else if ((b_over >> j) & 1u) {
                stop = j;
                undecided = true;
            } else {
                stop = j + 1;
                hit_max = true;
            }
        }
        const int lim = stop < 0 ? nvalid : stop;
        if (lane < lim) {
            const bool a = (accm >> lane) & 1u;
            const int rank = k + __popc(accm & ((1u << lane) - 1u));
            acc_s[UG_IDX(r, kSmaxCap)] = a ? rank : -1;
            gid_s[UG_IDX(r, kSmaxCap)] = a ? (int32_t)(c.n_slots + rank) : -1;
        }
        __syncwarp();
        const uint32_t taken = accm & (lim >= 32 ? 0xffffffffu : ((1u << lim) - 1u));
        k += __popc(taken);
        n_unique += __popc(taken);
        if (stop >= 0) {
            stop_at = r0 + stop;
            break;
        }
    }
    // Group rounds, one survivor at a time.  The per-survivor data comes in ahead of its
    // step: contact counts and pre-round groups of 32 survivors at once (lane i holds
    // survivor r0 + i), and the next survivor's list while this one is decided.
    int w_cnt = 0;
    int32_t w_g0 = -1, nx0 = -1, nx1 = -1;
    auto load_window = [&](int rb) {
        const int rr = rb + lane;
        w_cnt = 0;
        w_g0 = -1;
        if (rr < S_eff) {
            w_cnt = d.ccount[UG_IDX(rr, d.S_max)];
            w_g0 = d.g0[UG_IDX(d.surv_off[UG_IDX(rr, d.S_max + 1)], d.B_max)];
        }
    };
    auto load_list = [&](int rr, int nn) {
        const int32_t* l = d.clist + UG_IDX((int64_t)rr * kConflictCap, (int64_t)d.S_max * kConflictCap);
        nx0 = lane < nn ? l[lane] : -1;
        nx1 = lane + 32 < nn ? l[lane + 32] : -1;
    };
    if (group && S_eff > 0) {
        load_window(0);
        load_list(0, min(__shfl_sync(0xffffffffu, w_cnt, 0), kConflictCap));
    }
    for (int r = 0; group && r < S_eff; r++) {
        if (k >= room) {
            stop_at = r;
            grow = true;
            break;
        }
        const int n_all = __shfl_sync(0xffffffffu, w_cnt, r & 31);
        const int32_t g0 = __shfl_sync(0xffffffffu, w_g0, r & 31);
        const bool over = n_all > kConflictCap;  // the list holds only kConflictCap contacts
        const int n = over ? kConflictCap : n_all;
        const int32_t e0 = nx0, e1 = nx1;  // this survivor's list entries lane, lane + 32
        if (r + 1 < S_eff) {
            if (((r + 1) & 31) == 0) load_window(r + 1);
            load_list(r + 1, min(__shfl_sync(0xffffffffu, w_cnt, (r + 1) & 31), kConflictCap));
        }
        bool accept;
        int32_t gid;
        // union of the pre-round group and the groups of admitted earlier survivors
        int32_t mine = -1;
        bool two = false;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int32_t e = h ? e1 : e0;
            if (lane + 32 * h < n) {
                const int r2 = (int)UG_IDX(e, kSmaxCap);
                if (acc_s[r2] >= 0) {
                    const int32_t g2 = gid_s[r2];
                    if (mine == -1)
                        mine = g2;
                    else if (mine != g2)
                        two = true;
                }
            }
        }
        // the first group in list order: the pre-round one, else the lowest lane's
        const uint32_t hasg = __ballot_sync(0xffffffffu, mine != -1);
        int32_t first = g0;  // g0 and hasg are the same in every lane
        if (first == -1 && hasg) first = __shfl_sync(0xffffffffu, mine, __ffs(hasg) - 1);
        two = two || (mine != -1 && mine != first);
        two = __any_sync(0xffffffffu, two);
        if (!two && over) {  // unlisted contacts might add a group: decide next round
            stop_at = r;
            undecided = true;
            break;
        }
        if (two) {
            accept = false;
            gid = -1;
        } else if (first == -1) {
            accept = unique_group;  // touches nothing: founds a group, or (subpath) rejected
            gid = (int32_t)(c.n_slots + k);
        } else {
            accept = true;
            gid = first;
        }
        if (lane == 0) {
            acc_s[UG_IDX(r, kSmaxCap)] = accept ? k : -1;
            gid_s[UG_IDX(r, kSmaxCap)] = accept ? gid : -1;
        }
        __syncwarp();
        if (accept) {
            k++;
            if (!group || (unique_group && gid == (int32_t)(c.n_slots + k - 1)))
                n_unique++;
            else
                n_sub++;
            if (c.phase == 1 && c.max_n > 0 && n_unique >= c.max_n) {
                stop_at = r + 1;
                hit_max = true;
                break;
            }
        }
    }
    for (int r = lane; r < S; r += 32) {
        d.acc_rank[UG_IDX(r, d.S_max)] = r < stop_at ? acc_s[UG_IDX(r, kSmaxCap)] : -1;
        d.sgid[UG_IDX(r, d.S_max)] = r < stop_at ? gid_s[UG_IDX(r, kSmaxCap)] : -1;
    }
    if (lane != 0) return;
    int64_t next;
    if (hit_max)
        next = c.round_base + d.surv_off[UG_IDX(stop_at - 1, d.S_max + 1)] + 1;
    else if (stop_at < c.S_raw)
        next = c.round_base + d.surv_off[UG_IDX(stop_at, d.S_max + 1)];
    else
        next = c.round_base + c.B;
    const int64_t used = next - c.round_base;
    c.stop_at = stop_at;
    c.n_slots_prev = c.n_slots;
    c.n_slots += k;
    c.n_unique = n_unique;
    c.n_sub = n_sub;
    c.accepted_round = k;
    c.next_cand = next;
    c.attempts = next;
    c.last_used = used;
    c.rounds++;
    if (grow) c.state = ST_GROW;
    // round-size adaptation (the reference steers toward 64..512 survivors for
    // its serial host admission, braid_cuda.cu:921-924; the device resolver
    // takes up to S_max, so steer toward the survivor capacity instead).
    // Admission results do not depend on it.
    if (undecided && c.round_B > kTile)  // crowded in-round contacts: smaller rounds
        c.round_B = max(c.round_B >> 1, kTile);
    else if (c.S_raw > d.S_max && c.round_B > c.B_min)
        c.round_B = max(c.round_B >> 1, c.B_min);
    else if (c.S_raw < d.S_max / 4 && c.round_B < c.B_cap)
        c.round_B = min(c.round_B << 1, c.B_cap);
}

// ---------------------------------------------------------------- commit

// Appends slot to the chain of cell lin at timestep t; *old_head gets the
// previous head.  *new_key is set when the insert claimed a new hash key (the
// caller counts them into UniCtl::hash_used).
__device__ __forceinline__ void grid_insert(const UniDev& d, UniCtl& c, int t, int64_t lin, uint32_t fbit,
                                            int64_t cpt, int32_t slot, int32_t* old_head, bool* new_key,
                                            bool* new_cell) {
    if (d.grid_kind == GRID_DENSE) {
        *old_head = atomicExch(d.heads + UG_IDX((int64_t)t * cpt + lin, d.dense_cells), slot);
        *new_cell = *old_head < 0;
        return;
    }
    const uint64_t key = ((uint64_t)t << 40) | (uint64_t)lin;
    uint64_t h = mix64(key) & d.hmask;
    for (uint64_t probe = 0; probe <= d.hmask; probe++) {
        unsigned long long* kp = &d.hslot[h].x;
        const ulonglong2 sv = __ldcg(&d.hslot[h]);  // key and y in one load
        uint64_t k = sv.x;
        if (k == kEmptyKey) {
            const uint64_t prev = atomicCAS(kp, kEmptyKey, key);
            if (prev == kEmptyKey) {
                *new_key = true;
                k = key;
            } else {
                k = prev;
            }
        }
        if (k == key) {
            // y: chain head (low half), complemented cell mask of a coarse key (high half)
            if (!fbit) {
                *old_head = (int32_t)atomicExch(reinterpret_cast<unsigned int*>(&d.hslot[h].y), (unsigned int)slot);
                *new_cell = *old_head < 0;
                return;
            }
            // coarse key: the new head and the cell's bit in one compare-and-swap of y
            // (a failed swap means another insert into this coarse cell went first)
            unsigned long long* yp = &d.hslot[h].y;
            unsigned long long cur = sv.y;
            for (int it = 0; it < (1 << 20); it++) {
                const unsigned long long nv = (((cur >> 32) & ~(unsigned long long)fbit) << 32) | (uint32_t)slot;
                const unsigned long long prev = atomicCAS(yp, cur, nv);
                if (prev == cur) {
                    *old_head = (int32_t)(uint32_t)cur;
                    *new_cell = ((cur >> 32) & fbit) != 0ull;
                    return;
                }
                cur = prev;
            }
            break;
        }
        h = (h + 1) & d.hmask;
    }
    *old_head = -1;
    *new_cell = false;
    c.err_code = 3;  // hash full (host keeps the load factor below 1/2), or no progress
    c.state = ST_ERROR;
}

// Sets a bit of an occupancy bitmap; bits are only ever set during a run, so
// a bit read as set needs no atomic (most are: an unconditional atomicOr took
// k_commit from 56 to 63 ms per c3 job).
__device__ __forceinline__ void occ_set(uint32_t* words, int64_t bit, int64_t nwords) {
    uint32_t* w = words + UG_IDX(bit >> 5, nwords);
    const uint32_t m = 1u << (bit & 31);
    if (!(__ldcg(w) & m)) atomicOr(w, m);
}

__device__ __forceinline__ void occ_set_mask(uint32_t* words, int64_t w, uint32_t m, int64_t nwords) {
    uint32_t* p = words + UG_IDX(w, nwords);
    if ((__ldcg(p) & m) != m) atomicOr(p, m);
}

// Dilated filter: marks every block holding a cell that meets the cube of
// half-width occ1_reach around the committed point x (cells wrap around the
// torus; per axis at most 5 cells, so at most 5 blocks).
__device__ __forceinline__ void occ1_mark(const UniDev& d, int t, const double* x) {
    int bk[3][5], nb[3] = {1, 1, 1};
#pragma unroll
    for (int ax = 0; ax < 3; ax++) {
        bk[ax][0] = 0;
        if (ax >= d.dim) continue;
        const int c0 = (int)floor((x[ax] - d.occ1_reach + 1.0) / d.cell);
        const int c1 = (int)floor((x[ax] + d.occ1_reach + 1.0) / d.cell);
        int n = 0;
        for (int c = c0; c <= c1 && n < 5; c++) {
            int w = c % d.gw;
            w += w < 0 ? d.gw : 0;
            const int b = w >> d.occ1_shift;
            bool seen = false;
            for (int k = 0; k < n; k++) seen |= bk[ax][k] == b;
            if (!seen) bk[ax][n++] = b;
        }
        nb[ax] = n;
    }
    // along the last axis the blocks are neighbouring bits: one masked update per word
    const int L = d.dim - 1;
    const int64_t t0 = (int64_t)t * d.occ1_per_t;
    for (int i0 = 0; i0 < (L > 0 ? nb[0] : 1); i0++)
        for (int i1 = 0; i1 < (L > 1 ? nb[1] : 1); i1++) {
            int64_t row = 0;
            if (L > 0) row = bk[0][i0];
            if (L > 1) row = row * d.occ1_gw + bk[1][i1];
            row = t0 + row * d.occ1_gw;
            int64_t wcur = -1;
            uint32_t m = 0;
            for (int i = 0; i < nb[L]; i++) {
                const int64_t bit = row + bk[L][i];
                if ((bit >> 5) != wcur) {
                    if (m) occ_set_mask(d.occ1, wcur, m, d.occ1_words);
                    wcur = bit >> 5;
                    m = 0;
                }
                m |= 1u << (bit & 31);
            }
            occ_set_mask(d.occ1, wcur, m, d.occ1_words);
        }
}

__global__ void __launch_bounds__(256) k_commit(const UniDev* __restrict__ U, UniCtl* ctl,
                                                RoundInfo* info) {
    const int n_uni = info->n_uni, total = info->total_spt;
    const int lane = threadIdx.x & 31;
    // items: (survivor, timestep) pairs, survivor-major per universe; the trip
    // count is uniform over the block so the warp-level counting below converges
    for (int w0 = blockIdx.x * blockDim.x; w0 < total; w0 += gridDim.x * blockDim.x) {
        const int w = w0 + threadIdx.x;
        int u = -1;
        bool new_key = false, new_cell = false;
        if (w < total) {
            u = find_uni(info->spt_off, n_uni, w);
            const UniDev& d = U[u];
            UniCtl& c = ctl[u];
            const int local = w - info->spt_off[u];
            const int r = local / d.T, t = local - r * d.T;
            const int k = r < c.stop_at ? d.acc_rank[UG_IDX(r, d.S_max)] : -1;
            if (k >= 0) {
                const int64_t slot = UG_IDX(c.n_slots_prev + k, d.slot_cap);
                Pt64 q = d.spos[UG_IDX((int64_t)r * d.T + t, (int64_t)d.S_max * d.T)];
                int cc[3] = {0, 0, 0};
#pragma unroll
                for (int ax = 0; ax < 3; ax++)
                    if (ax < d.dim) cc[ax] = cell_of(q.c[ax], d.cell, d.gw);
                int32_t old;
                uint32_t fbit;
                const int64_t lin = grid_lin(d, cc, &fbit);
                grid_insert(d, c, t, lin, fbit, cells_per_t(d), (int32_t)slot, &old, &new_key, &new_cell);
                occ_set(d.occ, occ_bit(d, t, cc), d.occ_words);
                occ1_mark(d, t, q.c);
                q.next = old;
                q.gid = d.sgid[UG_IDX(r, d.S_max)];
                d.pts[UG_IDX(slot * d.T + t, d.slot_cap * d.T)] = q;
                Pt32 f;
                f.c[0] = (float)q.c[0];
                f.c[1] = (float)q.c[1];
                f.c[2] = (float)q.c[2];
                f.next = old;
                d.ptf[UG_IDX(slot * d.T + t, d.slot_cap * d.T)] = f;
                if (t == 0)
                    d.acc_idx[UG_IDX(slot, d.slot_cap)] = c.round_base + d.surv_off[UG_IDX(r, d.S_max + 1)];
            }
        }
        // new hash keys and newly occupied cells: one atomic per (warp, universe)
        const uint32_t nk = __ballot_sync(0xffffffffu, new_key);
        const uint32_t ncl = __ballot_sync(0xffffffffu, new_cell);
        if (nk | ncl) {
            const uint32_t peers = __match_any_sync(0xffffffffu, u);
            const uint32_t mine = nk & peers, minec = ncl & peers;
            if (new_key && lane == __ffs(mine) - 1)
                atomicAdd((unsigned long long*)&ctl[u].hash_used, (unsigned long long)__popc(mine));
            if (new_cell && lane == __ffs(minec) - 1)
                atomicAdd((unsigned long long*)&ctl[u].round_new, (unsigned long long)__popc(minec));
        }
    }
}

// Rebuild the main-grid hash of universe u from its committed points (after
// the host swapped in a larger, empty table).
__global__ void k_rehash(const UniDev* __restrict__ U, UniCtl* ctl, int u, int64_t n_slots) {
    const UniDev& d = U[u];
    UniCtl& c = ctl[u];
    const int64_t total = n_slots * d.T;
    for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < total;
         w += (int64_t)gridDim.x * blockDim.x) {
        const int64_t slot = w / d.T;
        const int t = (int)(w % d.T);
        Pt64* q = d.pts + slot * d.T + t;
        int cc[3] = {0, 0, 0};
#pragma unroll
        for (int ax = 0; ax < 3; ax++)
            if (ax < d.dim) cc[ax] = cell_of(q->c[ax], d.cell, d.gw);
        int32_t old;
        bool new_key = false, new_cell = false;
        uint32_t fbit;
        const int64_t lin = grid_lin(d, cc, &fbit);
        grid_insert(d, c, t, lin, fbit, cells_per_t(d), (int32_t)slot, &old, &new_key, &new_cell);
        if (new_key) atomicAdd((unsigned long long*)&c.hash_used, 1ull);
        q->next = old;
        d.ptf[slot * d.T + t].next = old;
    }
}

}  // namespace ug

namespace ug {

// Worldline parameters in term order (the --dump-params content): knot mode
// replays the reference draw sequence (cuda/braid_knot.cu:111-166) keeping
// each term; the Philox stream lists term j = frequency j + 2.
__global__ void k_params(const UniDev* __restrict__ U, int u, int64_t n, double* a2o, double* ao,
                         int32_t* bo, double* fo) {
    const UniDev& d = U[u];
    const int D = d.dim, nw = d.nw, F = d.F;
    double wj[kMaxF];
    int32_t bj[kMaxF];
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < n;
         s += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t idx = (uint64_t)d.acc_idx[s];
        if (d.rng == RNG_KNOT) {
            Xo r;
            r.seed(knot_seed(d.seed, idx));
            for (int ax = 0; ax < D; ax++) {
                const int64_t o = (s * D + ax) * nw;
                if ((uint32_t)nw == d.modmax) {
                    for (int j = 0; j < nw; j++) bj[j] = j + 2;
                    for (int j = nw - 1; j > 0; j--) {
                        const int k = (int)r.below((uint32_t)(j + 1));
                        const int32_t tmp = bj[j];
                        bj[j] = bj[k];
                        bj[k] = tmp;
                    }
                } else {
                    for (int j = 0; j < nw; j++) {
                        int bnew = 0;
                        bool dup = true;
                        for (int guard = 0; dup && guard < 64; guard++) {
                            bnew = (int)r.below(d.modmax) + 2;
                            dup = false;
                            for (int k = 0; k < j; k++)
                                if (bj[k] == bnew) dup = true;
                        }
                        bj[j] = bnew;
                    }
                }
                double sum = 0.0;
                for (int j = 0; j < nw; j++) {
                    wj[j] = -log(1.0 - r.f64());
                    sum += wj[j];
                }
                for (int j = 0; j < nw; j++) wj[j] /= sum;
                for (int j = 0; j < nw; j++) {
                    double amp = wj[j] / (double)bj[j];
                    if (r.flip()) amp = -amp;
                    ao[o + j] = amp;
                    bo[o + j] = bj[j];
                    fo[o + j] = (bj[j] % 2 == 0) ? r.f64() * kPi : 0.0;
                }
                a2o[s * D + ax] = d.pin ? 0.0 : (r.f64() * 2.0 - 1.0);
            }
        } else {
            for (int ax = 0; ax < D; ax++) {
                const int64_t o = (s * D + ax) * nw;
                double sum = 0.0;
                for (int p = 0; 2 * p <= F; p++) {
                    const uint4 q = philox_block(d.seed, idx, ax, p);
                    if (p == 0) {
                        a2o[s * D + ax] = d.pin ? 0.0 : (double)q.x * (1.0 / 2147483648.0) - 1.0;
                        continue;
                    }
                    const int be = 2 * p, bo2 = 2 * p + 1;
                    const double Ee = -log(((double)q.x + 0.5) * (1.0 / 4294967296.0));
                    sum += Ee;
                    ao[o + be - 2] = (q.z & 1u) ? -Ee : Ee;
                    fo[o + be - 2] = (double)(q.z >> 1) * (1.0 / 2147483648.0) * kPi;
                    bo[o + be - 2] = be;
                    if (bo2 <= F) {
                        const double Eo = -log(((double)q.y + 0.5) * (1.0 / 4294967296.0));
                        sum += Eo;
                        ao[o + bo2 - 2] = (q.w & 1u) ? -Eo : Eo;
                        fo[o + bo2 - 2] = 0.0;
                        bo[o + bo2 - 2] = bo2;
                    }
                }
                for (int j = 0; j < nw; j++) {
                    const double e = ao[o + j];
                    double amp = fabs(e) / sum / (double)(j + 2);
                    ao[o + j] = e < 0.0 ? -amp : amp;
                }
            }
        }
    }
}

void launch_params(const UniDev* dU, int u, int64_t n, double* a2, double* a, int32_t* b, double* f,
                   cudaStream_t st) {
    const int blocks = (int)std::min<int64_t>((n + 127) / 128, 4096);
    k_params<<<blocks, 128, 0, st>>>(dU, u, n, a2, a, b, f);
}

// ------------------------------------------------------------- read-back

// Accepted candidate indices and group labels of every universe into one
// contiguous pair of arrays (universe u at [off[u], off[u+1])), so that a
// caller reads all of them back with one copy each.  One CTA per universe.
__global__ void k_gather_accepted(const UniDev* __restrict__ U, const int64_t* __restrict__ off,
                                  int64_t* __restrict__ idx, int32_t* __restrict__ gid) {
    const int u = blockIdx.x;
    const UniDev& d = U[u];
    const int64_t o = off[u], n = off[u + 1] - o;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        idx[o + i] = d.acc_idx[UG_IDX(i, d.slot_cap)];
        gid[o + i] = d.pts[UG_IDX(i * d.T, d.slot_cap * d.T)].gid;
    }
}

}  // namespace ug
