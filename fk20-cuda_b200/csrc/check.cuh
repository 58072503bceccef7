// check.cuh -- the checked build's index and range checks.
//
// `make checked` builds libfk20b200_checked.so with FK_CHECKED=1: the MSM and
// the persistent G1 FFT then test what they compute from their arguments
// (task decoding, tile and table indices, the signed-digit recoding's final
// carry) against the sizes they were given.  A failed check never traps: the
// kernel records the first failing site (FK20_CHECK_* codes) in a device word
// of its translation unit and skips the access.  fk20_check_status() returns
// and clears those words.  In the normal build the checks compile to nothing.
#pragma once
#include <cuda_runtime.h>

#ifndef FK_CHECKED
#define FK_CHECKED 0
#endif

// one word per translation unit that runs checks, plus its host accessor
#define FK_CHECK_WORD(tu)                                                       \
    static __device__ int g_check_##tu;                                        \
    int check_take_##tu() {                                                     \
        int v = 0, z = 0;                                                       \
        if (cudaMemcpyFromSymbol(&v, g_check_##tu, sizeof v) != cudaSuccess) {  \
            cudaGetLastError();                                                 \
            return 0;                                                           \
        }                                                                       \
        cudaMemcpyToSymbol(g_check_##tu, &z, sizeof z);                         \
        return v;                                                               \
    }

// true when `cond` holds; otherwise records `site` (first failure wins)
#if FK_CHECKED
#define FK_CHECK(word, cond, site) ((cond) ? true : (atomicCAS(&(word), 0, (site)), false))
#else
#define FK_CHECK(word, cond, site) true
#endif
