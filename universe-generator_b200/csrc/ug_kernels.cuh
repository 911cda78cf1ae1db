// ug_kernels.cuh -- declarations shared by the round-pipeline kernels and
// the host runtime.
#pragma once
#include "ug_device.cuh"

namespace ug {

constexpr int kMaxUni = 1024;

// Work decomposition of one round across all universes (device resident).
struct RoundInfo {
    int32_t n_uni;
    int32_t total_tiles;
    int32_t total_surv;
    int32_t compact_done;
    int32_t any_active;
    int32_t mixed_ok;      // universes in the mixed prefilter this round
    int32_t gemm_next;     // k_surv_gemm: product tiles handed out so far
    int32_t pad1;
    int32_t total_gray;
    int32_t gray_done;
    int32_t tile_next;     // mixed prefilter: tiles handed out beyond the first gridDim.x
    int32_t confl_next;    // k_conflicts: survivors handed out so far
    int32_t total_sev;     // k_surv_gemm warp tiles (32 rows x 32 timesteps)
    int32_t total_spt;     // survivor timesteps (k_surv_hash / k_commit items)
    int32_t tile_off[kMaxUni + 1];   // prefilter tiles: first tile of the i-th universe in tile order
    int32_t tile_uni[kMaxUni];       // the universe at position i of the tile order
    int32_t surv_off[kMaxUni + 1];
    int32_t surv_off_o[kMaxUni + 1];  // survivor offsets of the universes in tile order
    int32_t gray_pref[kMaxUni + 1];
    int32_t sev_off[kMaxUni + 1];
    int32_t sev_off_o[kMaxUni + 1];   // product tile offsets of the universes in tile order
    int32_t spt_off[kMaxUni + 1];
};

// Term k of the survivor product: sin term of frequency b at k = kseq_s(b),
// its cos term (even b) at kseq_s(b) + 1.
__host__ __device__ __forceinline__ int kseq_s(int b) { return (b - 2) + ((b - 1) >> 1); }
__host__ __device__ __forceinline__ int kseq_len(int F) { return kseq_s(F) + 1 + ((F & 1) ? 0 : 1); }

__device__ __forceinline__ int find_uni(const int32_t* off, int n, int item) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= item)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// Kernels (ug_kernels.cu)
__global__ void k_plan(const UniDev* __restrict__ U, UniCtl* ctl, RoundInfo* info);
__global__ void k_gray_compact(const UniDev* __restrict__ U, UniCtl* ctl, RoundInfo* info, int all);
// The FP64 test of undecided candidates (k_confirm64w, a template kept inside
// ug_kernels.cu): every candidate of the round (all = 1, a warp per candidate) or
// the mixed form's retest (all = 0, a block per candidate).
cudaError_t confirm64w_set_smem();
void launch_confirm64w(int all, int nsm, const UniDev* U, UniCtl* ctl, RoundInfo* info, cudaStream_t st);
__global__ void k_compact(const UniDev* __restrict__ U, UniCtl* ctl, RoundInfo* info);
__global__ void k_surv_gen(const UniDev* __restrict__ U, UniCtl* ctl, RoundInfo* info, int warp_bytes);
__global__ void k_surv_gemm(const UniDev* __restrict__ U, UniCtl* ctl, RoundInfo* info);
__global__ void k_surv_hash(const UniDev* __restrict__ U, UniCtl* ctl, RoundInfo* info);
__global__ void k_restore_gen(const UniDev* __restrict__ U, int u, const int64_t* __restrict__ idx, int m);
__global__ void k_probe(const UniDev* __restrict__ U, int u, int64_t n_slots, uint64_t seed, int64_t n, int bins,
                        unsigned long long* proposed, unsigned long long* accepted);
__global__ void k_conflicts(const UniDev* __restrict__ U, UniCtl* ctl, RoundInfo* info);
__global__ void k_greedy(const UniDev* __restrict__ U, UniCtl* ctl, RoundInfo* info);
__global__ void k_commit(const UniDev* __restrict__ U, UniCtl* ctl, RoundInfo* info);
__global__ void k_rehash(const UniDev* __restrict__ U, UniCtl* ctl, int u, int64_t n_slots);
__global__ void k_gather_accepted(const UniDev* __restrict__ U, const int64_t* __restrict__ off,
                                  int64_t* __restrict__ idx, int32_t* __restrict__ gid);

// k_surv_gemm: terms per shared-memory chunk; two stages of A and B per warp.
constexpr int kGemmKC = 8;
constexpr size_t kGemmSmem = (size_t)4 * 2 * 2 * kGemmKC * 32 * sizeof(double);  // 4 warps per CTA

// Shared memory of k_surv_gen per warp (bytes), for F <= kMaxF.
constexpr int kSurvWarps = 4;
constexpr size_t kSurvSmemPerWarpBase = (size_t)3 * (kMaxF + 1) * 2 * sizeof(double) + 3 * sizeof(double) +
                                    (size_t)kMaxF * (sizeof(int32_t) + sizeof(double));
constexpr size_t kSurvSmemPerWarp = kSurvSmemPerWarpBase;
// k_surv_gen on a batch without knot-stream universes: one axis of alpha / beta
constexpr size_t kSurvSmemAxis = (size_t)2 * (kMaxF + 1) * sizeof(double);
// k_confirm64w adds the FP64 trajectory of a 1+1D candidate
constexpr size_t kConfSmemPerWarp = kSurvSmemPerWarpBase + (size_t)kMaxF * sizeof(double);

}  // namespace ug
