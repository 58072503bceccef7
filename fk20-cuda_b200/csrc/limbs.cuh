// limbs.cuh -- qualifiers and single-word helpers for multi-limb integer
// arithmetic.
//
// The carry chains themselves (add.cc / addc / mad.lo.cc / madc.hi.cc ...)
// are not here: each chain is one inline-PTX statement in chains.inc, called
// through the ch_* functions of field.cuh, because the carry flag CC.CF is
// invisible to the compiler and must not cross from one asm statement to
// another.  Host builds of the field code (the library's host-side
// precomputation and the CPU unit tests) use portable stand-ins.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define FK_HD __host__ __device__ __forceinline__
#define FK_D __device__ __forceinline__
#else
#define FK_HD inline
#define FK_D inline
#endif

namespace fk {

FK_HD uint32_t mul_lo(uint32_t a, uint32_t b) { return a * b; }
FK_HD uint32_t mul_hi(uint32_t a, uint32_t b) {
#if defined(__CUDA_ARCH__)
    return __umulhi(a, b);
#else
    return (uint32_t)(((uint64_t)a * b) >> 32);
#endif
}

}  // namespace fk
