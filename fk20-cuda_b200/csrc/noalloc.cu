// noalloc.cu -- a G1 FFT entry point that never allocates device memory.
//
// Some callers cannot let a library call cudaMalloc: code whose device memory
// is entirely handed out by its own allocator or memory pool (a framework that
// reserves the GPU up front), latency-critical paths that must not take the
// implicit device-wide synchronisation of cudaMalloc/cudaFree, and callers that
// are not allowed to grow their device footprint after start-up.  For them,
// g1p_fft_noalloc runs the same batched G1 FFT as g1p_fft_n, but its working
// tiles live in one fixed, file-scope device array instead of a buffer
// allocated on first use.
//
// Limits and behaviour:
//  - at most NOALLOC_MAX_TRANSFORMS transforms of up to 512 points per call;
//    larger requests return FK20_ETOOBIG before anything is launched;
//  - the array (NOALLOC_TILE_BYTES, ~4.7 MB) is part of the library's device
//    image: every GPU that loads the library holds it until the process exits;
//  - the first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (with that device current) and caches it; make that
//    first call before any stream capture;
//  - all calls share the array and it keeps the previous call's contents.
//    Nothing has to start at zero: every tile a call reads was first written
//    by the same call (padding lanes are written as the point at infinity).
//    Calls that overlap on the GPU (different streams, or different host
//    threads without ordering) race on the array and corrupt each other's
//    results; serialise them.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/fk20_b200.h"
#include "launch.h"
#include "layout.cuh"

namespace fk {

constexpr unsigned NOALLOC_MAX_TRANSFORMS = 64;
constexpr size_t NOALLOC_TILE_UINT4 = (size_t)(NOALLOC_MAX_TRANSFORMS / 32) * 512 * TILE_Q * 32;
constexpr size_t NOALLOC_TILE_BYTES = NOALLOC_TILE_UINT4 * sizeof(uint4);

static __device__ __align__(256) uint4 g_noalloc_tiles[NOALLOC_TILE_UINT4];

int device_ready();  // engine.cu: constant tables of the current device

namespace {

std::mutex g_noalloc_mu;
uint4 *g_noalloc_ptr[64];

// device address of g_noalloc_tiles on the current device (looked up once)
int noalloc_tiles(uint4 **out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return FK20_ENODEV;
    }
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_tiles);
        if (e != cudaSuccess) return (int)e;
        g_noalloc_ptr[dev] = (uint4 *)p;
    }
    *out = g_noalloc_ptr[dev];
    return 0;
}

}  // namespace
}  // namespace fk

using namespace fk;

extern "C" int g1p_fft_noalloc(g1p_t *output, const g1p_t *input, unsigned log_m, unsigned count, int inverse,
                               void *stream) {
    if (!output || !input || log_m < 1 || log_m > 9 || count == 0) return FK20_EINVAL;
    if (((uintptr_t)output | (uintptr_t)input) & 15) return FK20_EINVAL;
    if (count > NOALLOC_MAX_TRANSFORMS) return FK20_ETOOBIG;
    int rc = device_ready();
    if (rc) return rc;
    uint4 *D = nullptr;
    rc = noalloc_tiles(&D);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const int G = (int)((count + 31) / 32);
    const int L = (int)log_m;
    if (!inverse) {  // bit-reversed load, forward DIT stages -> natural order
        launch_ref_to_tile(D, (const uint64_t *)input, (int)count, G, L, 1, 0, st);
        for (int s = 0; s < L; s++) launch_g1_stage(D, G, L, s, 1, st);
        launch_tile_to_ref((uint64_t *)output, D, nullptr, (int)count, L, 0, st);
    } else {  // natural load, inverse DIF stages -> bit-reversed, times 1/m
        launch_ref_to_tile(D, (const uint64_t *)input, (int)count, G, L, 0, 0, st);
        for (int s = 0; s < L; s++) launch_g1_stage(D, G, L, s, 0, st);
        launch_g1_scale(D, G, L, 512 + L, st);
        launch_tile_to_ref((uint64_t *)output, D, nullptr, (int)count, L, 1, st);
    }
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : (int)e;
}
