// consts.cuh -- device constant tables shared by every kernel translation unit.
//
// Each .cu file of the engine is its own (non-relocatable) CUDA module, so it
// holds its own copy of these tables; engine.cu uploads the host-computed
// values into every module once per device (fk_upload_consts_* below).
#pragma once
#include <cuda_runtime.h>
#include "scalar_prog.cuh"

namespace fk {

constexpr int MAX_LOG_M = 9;     // FFT sizes up to 512 (n = 4096, l = 16)
constexpr int NPROG = 512 + 16;  // w_512^t for t < 512, then 2^-s at index 512 + s
constexpr int L_COLS = 16;       // l: toeplitz columns per row (fk20_multi_cuda.py:328)

// fixed-scalar programs: read with warp-uniform addresses (one broadcast per load)
static __device__ uint32_t c_prog[NPROG][PROG_WORDS];
static __device__ uint32_t g_fr_tw[512][8];   // w_512^t * 2^256 mod r (Montgomery form)
static __device__ uint32_t g_fr_inv2[16][8];  // 2^-s * 2^256 mod r

struct HostConsts {
    uint32_t prog[NPROG][PROG_WORDS];
    uint32_t fr_tw[512][8];
    uint32_t fr_inv2[16][8];
    int prog_dbl[NPROG], prog_add[NPROG];
};

const HostConsts &host_consts();

static inline cudaError_t upload_module_consts() {
    const HostConsts &hc = host_consts();
    cudaError_t e = cudaMemcpyToSymbol(c_prog, hc.prog, sizeof(hc.prog));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_fr_tw, hc.fr_tw, sizeof(hc.fr_tw));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_fr_inv2, hc.fr_inv2, sizeof(hc.fr_inv2));
    return e;
}

}  // namespace fk
