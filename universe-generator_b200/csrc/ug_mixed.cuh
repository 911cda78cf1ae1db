// ug_mixed.cuh -- mixed-precision (tensor-core) prefilter interface.
#pragma once
#include <cuda_runtime.h>

#include "../../include/ug.h"
#include "ug_kernels.cuh"

namespace ug {

// Per-universe operand tables of the tensor-core evaluation.
struct MixedTables {
    void* bhi = nullptr;   // B operand (hi BF16), UMMA canonical layout
    void* blo = nullptr;   // B operand (lo BF16)
    int32_t K = 0;         // padded contraction length
    int32_t Tp = 0;        // padded timestep count
    double margin = 0.0;   // guard band applied to the FP32 Chebyshev test
};

int mixed_setup(const ug_universe_cfg& cfg, UniDev& d, MixedTables& mt);
void mixed_free(MixedTables& mt);
int mixed_init_kernels();
void launch_prefilter_mixed(const UniDev* dU, UniCtl* dCtl, RoundInfo* dInfo, int nsm, bool any_group,
                            bool any_euclid, cudaStream_t st);
int mixed_error(const UniDev* dU, int u, const UniDev& d, const MixedTables& mt, int64_t first,
                int64_t count, double* max_err, double* margin, double* max_ratio, cudaStream_t st);
void launch_params(const UniDev* dU, int u, int64_t n, double* a2, double* a, int32_t* b, double* f,
                   cudaStream_t st);
// Runs k_wait_selftest on the current device; *status gets its result.
int wait_selftest(int64_t limit_ns, int32_t* status);

}  // namespace ug
