// ug_noalloc.cu -- parameter dump that allocates no device memory.
//
// ug_batch_params stages the regenerated worldline parameters in device
// buffers it allocates for the call.  Some callers cannot call cudaMalloc at
// that point: a serving process that reserved all of its device memory when
// it started and runs with none to spare, or a host whose allocator policy
// forbids allocations outside start-up.  For them,
// ug_batch_params_noalloc stages the same kernel's output in one fixed
// buffer that lives in the library image: a file-scope __device__ array of
// kStageBytes (16 MiB), present on every GPU that loads the library until
// the process exits.  Dumps larger than that are rejected with UG_ECAP.
//
// The array is shared by every call: each call overwrites the part it uses
// (nothing needs to start at zero), and calls whose kernels overlap on the
// GPU race on it.  Host code cannot pass the array's name to a kernel (on
// the host it is only a stand-in symbol), so the first call on each device
// looks up its device address with cudaGetSymbolAddress, with that device
// current, and caches it; make that first call before any stream capture.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <mutex>

#include "../../include/ug.h"
#include "ug_kernels.cuh"
#include "ug_mixed.cuh"

namespace ug {

int batch_params_view(void* h, int u, const UniDev** dU, int64_t* n, int* dim, int* nw, int* dev,
                      cudaStream_t* st);
int set_error(int code, const char* msg);

constexpr size_t kStageBytes = (size_t)16 << 20;
static __device__ __align__(256) unsigned char g_param_stage[kStageBytes];

constexpr int kMaxDevices = 64;
static void* g_stage_addr[kMaxDevices];
static std::mutex g_stage_mu;

// Device address of g_param_stage on the current device (looked up once).
static int stage_address(int dev, void** out) {
    if (dev < 0 || dev >= kMaxDevices) return set_error(UG_EINVAL, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_stage_mu);
    if (!g_stage_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_param_stage);
        if (e != cudaSuccess) {
            char msg[256];
            snprintf(msg, sizeof msg, "cudaGetSymbolAddress(parameter stage): %s", cudaGetErrorString(e));
            return set_error(UG_ECUDA, msg);
        }
        g_stage_addr[dev] = p;
    }
    *out = g_stage_addr[dev];
    return UG_OK;
}

}  // namespace ug

using namespace ug;

extern "C" int ug_batch_params_noalloc(void* h, int32_t u, double* a2, double* a, int32_t* b, double* f,
                                       int64_t cap_paths) {
    const UniDev* dU = nullptr;
    int64_t n = 0;
    int dim = 0, nw = 0, dev = 0;
    cudaStream_t st = nullptr;
    int rc = batch_params_view(h, u, &dU, &n, &dim, &nw, &dev, &st);
    if (rc) return rc;
    if (cap_paths < n) return set_error(UG_ECAP, "params buffer too small");
    if (n == 0) return UG_OK;
    // layout in the stage: a2 [n][dim] f64 | a [n][dim][nw] f64 | f [..] f64 | b [..] i32
    const size_t n_a2 = (size_t)n * dim, n_t = (size_t)n * dim * nw;
    const size_t bytes = n_a2 * 8 + n_t * 8 * 2 + n_t * 4;
    if (bytes > kStageBytes) {
        char msg[256];
        snprintf(msg, sizeof msg,
                 "parameter dump of %lld paths needs %zu bytes; the fixed stage holds %zu (use ug_batch_params)",
                 (long long)n, bytes, kStageBytes);
        return set_error(UG_ECAP, msg);
    }
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess) return set_error(UG_ECUDA, "cudaGetDevice failed");
    if (cur != dev && cudaSetDevice(dev) != cudaSuccess) return set_error(UG_ECUDA, "cudaSetDevice failed");
    void* stage = nullptr;
    rc = stage_address(dev, &stage);
    if (rc == UG_OK) {
        unsigned char* s = (unsigned char*)stage;
        double* da2 = (double*)s;
        double* da = (double*)(s + n_a2 * 8);
        double* df = (double*)(s + n_a2 * 8 + n_t * 8);
        int32_t* db = (int32_t*)(s + n_a2 * 8 + n_t * 16);
        launch_params(dU, u, n, da2, da, db, df, st);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess && a2) e = cudaMemcpyAsync(a2, da2, n_a2 * 8, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess && a) e = cudaMemcpyAsync(a, da, n_t * 8, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess && f) e = cudaMemcpyAsync(f, df, n_t * 8, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess && b) e = cudaMemcpyAsync(b, db, n_t * 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            char msg[256];
            snprintf(msg, sizeof msg, "params (no-alloc): %s", cudaGetErrorString(e));
            rc = set_error(UG_ECUDA, msg);
        }
    }
    if (cur != dev) cudaSetDevice(cur);
    return rc;
}
