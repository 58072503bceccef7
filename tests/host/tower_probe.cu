// Test probe of the pairing's tower arithmetic (fk20-cuda_b200/csrc/tower.cuh):
// the sparse product of an Fp12 element by a Miller-loop line, computed in two
// code arrangements behind a plain C entry point (tests only).
//
//   variant 0: the library's f12_mul_line (its Fp6 sums written out);
//   variant 1: the same product with the Fp6 sums as the rolled
//              (#pragma unroll 1) loops of f6_add / f6_sub, placed after the
//              out-of-line Fp2 products.
//
// Both must equal the restatement's product.  Variant 1 is the arrangement
// that once gave wrong odd coefficients on the GPU while the carry chains of
// the field code were separate one-instruction asm statements.
#define FK_FP_MUL_OUTLINE 1
#include "../../fk20-cuda_b200/csrc/tower.cuh"

using namespace fk;

static __device__ __noinline__ void f12_mul_line_rolled(Fp12 *f, const Fp2 *l) {
    Fp6 t0, t1, s;
    Fp2 c23;
    f6_mul01(t0, f->a0, l[0], l[1]);
    f6_mul1(t1, f->a1, l[2]);
    f6_add(s, f->a0, f->a1);
    f2_add(c23, l[1], l[2]);
    f6_mul01(s, s, l[0], c23);
    f6_sub(s, s, t0);
    f6_sub(f->a1, s, t1);
    f6_mulv(t1, t1);
    f6_add(f->a0, t0, t1);
}

// f: n Fp12 values, l: n lines (c0, c2, c3), all Montgomery-form 32-bit words
// in the structs' order; f is overwritten with f * line
__global__ void k_line(int variant, Fp12 *f, const Fp2 *l, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Fp12 x = f[i];
    Fp2 ln[3] = {l[3 * i], l[3 * i + 1], l[3 * i + 2]};
    if (variant == 0)
        f12_mul_line(&x, ln);
    else
        f12_mul_line_rolled(&x, ln);
    f[i] = x;
}

extern "C" int tower_line(int variant, void *f, const void *l, int n) {
    k_line<<<(n + 63) / 64, 64>>>(variant, static_cast<Fp12 *>(f), static_cast<const Fp2 *>(l), n);
    return (int)cudaDeviceSynchronize();
}
