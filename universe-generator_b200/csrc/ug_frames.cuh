// ug_frames.cuh -- frame baking entry points shared with the host runtime.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/ug.h"

namespace ug {

// Largest frequency of device-resident dump parameters b[0..m) (work on stream st).
int max_b_device(const int32_t* b, int64_t m, int* out, cudaStream_t st);

// Frames of n device-resident 2+1 paths in dump layout: a2 [n][2], a/b/f [n][2][nw];
// every kernel and copy is issued on stream st.
int frames_from_params(const ug_frames_cfg* cfg, int n, int nw, int bMax, const double* dA2, const double* dA,
                       const int32_t* dBi, const double* dF, ug_frames_out* out, cudaStream_t st);

}  // namespace ug
