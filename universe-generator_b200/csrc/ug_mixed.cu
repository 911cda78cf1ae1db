// ug_mixed.cu -- mixed-precision prefilter (placeholder until the tensor-core path lands).
#include "ug_mixed.cuh"

namespace ug {

int mixed_setup(const ug_universe_cfg&, UniDev&, MixedTables&) { return UG_ENOTSUP; }
void mixed_free(MixedTables&) {}
int mixed_init_kernels() { return UG_OK; }
void launch_prefilter_mixed(const UniDev*, UniCtl*, RoundInfo*, int, cudaStream_t) {}
int mixed_error(const UniDev*, int, const UniDev&, const MixedTables&, int64_t, int64_t, double*,
                double*, cudaStream_t) {
    return UG_ENOTSUP;
}

}  // namespace ug
