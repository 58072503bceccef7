// kernels_misc.cu -- batched forms of the fp_* / fr_* / g1p_* device API
// (fp.cuh:16-41, fr.cuh:33-58, g1.cuh:31-96), the comparison / affine helpers
// (fr.cu:99, g1p.cu:142, g1p.cu:168), the Montgomery-product microbenchmark and
// the device-side fingerprint that keys cached tables.
#include "consts.cuh"
#include "launch.h"
#include "layout.cuh"

namespace fk {

cudaError_t upload_consts_misc() { return upload_module_consts(); }

template <class F>
__device__ void load_ref(Elem<F> &e, const uint64_t *x) {
#pragma unroll
    for (int k = 0; k < F::N / 2; k++) { e.w[2 * k] = (uint32_t)x[k]; e.w[2 * k + 1] = (uint32_t)(x[k] >> 32); }
}
template <class F>
__device__ void store_ref(uint64_t *x, const Elem<F> &e) {
#pragma unroll
    for (int k = 0; k < F::N / 2; k++) x[k] = (uint64_t)e.w[2 * k] | ((uint64_t)e.w[2 * k + 1] << 32);
}

template <class F>
__global__ void k_field_op(int op, uint64_t *out, const uint64_t *a, const uint64_t *b, size_t count) {
    constexpr int L = F::N / 2;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < count; e += (size_t)gridDim.x * blockDim.x) {
        Elem<F> x, y, z, t;
        load_ref(t, a + L * e);
        f_to_mont(x, t);
        if (b) { load_ref(t, b + L * e); f_to_mont(y, t); } else { f_set_zero(y); }
        switch (op) {
        case 0: f_mul(z, x, y); break;
        case 1: f_sqr(z, x); break;
        case 2: f_add(z, x, y); break;
        case 3: f_sub(z, x, y); break;
        case 4: f_neg(z, x); break;
        case 5: f_inv(z, x); break;
        case 7: f_dbl(z, x); break;
        case 8: f_dbl(z, x); f_add(z, z, x); break;
        case 9: f_dbl(z, x); f_dbl(z, z); break;
        case 10: f_dbl(z, x); f_dbl(z, z); f_dbl(z, z); break;
        case 11: f_mul12(z, x); break;
        default: z = x; break;  // 6: canonical reduction
        }
        f_from_mont(t, z);
        store_ref(out + L * e, t);
    }
}

// Y^2 Z == X^3 + 4 Z^3, or infinity (0, Y != 0, 0)   (g1p_ispoint.cu:14-60)
__device__ bool g1_on_curve(const G1P &p) {
    if (f_is_zero(p.z)) return !f_is_zero(p.y) && f_is_zero(p.x);
    Fp l, r, t;
    f_sqr(l, p.y);
    f_mul(l, l, p.z);
    f_sqr(r, p.x);
    f_mul(r, r, p.x);
    f_sqr(t, p.z);
    f_mul(t, t, p.z);
    f_dbl(t, t);
    f_dbl(t, t);
    f_add(r, r, t);
    return f_eq(l, r);
}

// double-and-add over a 256-bit scalar (g1p_mul.cu:18-67 semantics; any curve point)
__device__ void g1_mul_scalar(G1P &r, const G1P &p, const uint64_t *k) {
    G1P acc;
    g1_set_inf(acc);
    for (int i = 255; i >= 0; i--) {
        g1_dbl(acc, acc);
        if ((k[i >> 6] >> (i & 63)) & 1) g1_add(acc, acc, p);
    }
    r = acc;
}

__global__ void k_g1_op(int op, uint64_t *out, const uint64_t *a, const void *bv, size_t count) {
    const uint64_t *b = (const uint64_t *)bv;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < count; e += (size_t)gridDim.x * blockDim.x) {
        G1P p, q, r;
        if (op == 6) {  // raw coordinates: (X, Y, 0) is a point only with X = 0, Y != 0
            Fp t;
            load_ref(t, a + 18 * e); f_to_mont(p.x, t);
            load_ref(t, a + 18 * e + 6); f_to_mont(p.y, t);
            load_ref(t, a + 18 * e + 12); f_to_mont(p.z, t);
            ((uint8_t *)bv)[e] = g1_on_curve(p) ? 1 : 0;
            continue;
        }
        g1p_from_ref(p, a + 18 * e);
        switch (op) {
        case 0: g1p_from_ref(q, b + 18 * e); g1_add(r, p, q); break;
        case 1: g1_dbl(r, p); break;
        case 2: g1_neg(r, p); break;
        case 3: g1p_from_ref(q, b + 18 * e); g1_neg(q, q); g1_add(r, p, q); break;
        case 4: g1_mul_scalar(r, p, b + 4 * e); break;
        case 5: r = p; g1_normalize(r); break;
        default: r = p; break;
        }
        g1p_to_ref(out + 18 * e, r);
    }
}

__global__ void k_fr_eq(uint8_t *eq, const uint64_t *x, const uint64_t *y, size_t count) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < count; e += (size_t)gridDim.x * blockDim.x) {
        Fr a, b;
        fr_from_ref(a, x + 4 * e);
        fr_from_ref(b, y + 4 * e);
        eq[e] = f_eq(a, b) ? 1 : 0;
    }
}

// cross-multiplied equality, valid for infinity too (g1p_compare.cu:23-56)
__global__ void k_g1p_eq(uint8_t *eq, const uint64_t *pp, const uint64_t *qq, size_t count) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < count; e += (size_t)gridDim.x * blockDim.x) {
        G1P p, q;
        g1p_from_ref(p, pp + 18 * e);
        g1p_from_ref(q, qq + 18 * e);
        Fp a, b, c, d;
        f_mul(a, p.x, q.z);
        f_mul(b, q.x, p.z);
        f_mul(c, p.y, q.z);
        f_mul(d, q.y, p.z);
        eq[e] = (f_eq(a, b) && f_eq(c, d)) ? 1 : 0;
    }
}

__global__ void k_g1a_from_g1p(uint64_t *aout, const uint64_t *pin, size_t count) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < count; e += (size_t)gridDim.x * blockDim.x) {
        G1P p;
        g1p_from_ref(p, pin + 18 * e);
        Fp x, y;
        if (f_is_zero(p.z)) {
            f_set_zero(x);
            f_set_zero(y);
        } else {
            g1_normalize(p);
            f_from_mont(x, p.x);
            f_from_mont(y, p.y);
        }
        store_ref(aout + 12 * e, x);
        store_ref(aout + 12 * e + 6, y);
    }
}

// `iters` dependent Montgomery products per element, limb-major data
template <class F>
__global__ void k_bench_field(uint32_t *data, size_t count, int iters, int sqr) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < count; e += (size_t)gridDim.x * blockDim.x) {
        Elem<F> x, y;
#pragma unroll
        for (int k = 0; k < F::N; k++) x.w[k] = data[k * count + e];
        y = x;
        if (sqr) {
            for (int it = 0; it < iters; it++) f_sqr(x, x);
        } else {
            for (int it = 0; it < iters; it++) f_mul(x, x, y);
        }
#pragma unroll
        for (int k = 0; k < F::N; k++) data[k * count + e] = x.w[k];
    }
}

// order-sensitive 64-bit fingerprint of n words
__global__ void k_fingerprint(unsigned long long *out, const uint64_t *w, size_t n) {
    unsigned long long acc = 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        unsigned long long z = (unsigned long long)i * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        acc += (w[i] ^ (w[i] >> 29)) * (z | 1ull);
    }
    atomicAdd(out, acc);
}

// IMAD-pipe peak: 8 independent 32-bit multiply-add chains per thread
__global__ void k_bench_imad(uint32_t *sink, int iters, uint32_t b, uint32_t c) {
    uint32_t a[8];
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = threadIdx.x + k * 7919u + blockIdx.x;
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int u = 0; u < 4; u++) {
#pragma unroll
            for (int k = 0; k < 8; k++) a[k] = a[k] * b + c;
        }
    }
    uint32_t r = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) r ^= a[k];
    if (r == 0x9e3779b9u) sink[0] = r;  // keeps the chains live
}

void launch_bench_imad(uint32_t *sink, int blocks, int threads, int iters, cudaStream_t st) {
    k_bench_imad<<<blocks, threads, 0, st>>>(sink, iters, 0x01000193u, 0x811c9dc5u);
}

void launch_field_op(int field, int op, uint64_t *out, const uint64_t *a, const uint64_t *b, size_t count,
                     cudaStream_t st) {
    if (field == 0) k_field_op<FpDesc><<<grid_stride_blocks(count), 256, 0, st>>>(op, out, a, b, count);
    else k_field_op<FrDesc><<<grid_stride_blocks(count), 256, 0, st>>>(op, out, a, b, count);
}
void launch_g1_op(int op, uint64_t *out, const uint64_t *a, const void *b, size_t count, cudaStream_t st) {
    k_g1_op<<<grid_stride_blocks(count), 128, 0, st>>>(op, out, a, b, count);
}
void launch_fr_eq(uint8_t *eq, const uint64_t *x, const uint64_t *y, size_t count, cudaStream_t st) {
    k_fr_eq<<<grid_stride_blocks(count), 256, 0, st>>>(eq, x, y, count);
}
void launch_g1p_eq(uint8_t *eq, const uint64_t *p, const uint64_t *q, size_t count, cudaStream_t st) {
    k_g1p_eq<<<grid_stride_blocks(count), 128, 0, st>>>(eq, p, q, count);
}
void launch_g1a_from_g1p(uint64_t *a, const uint64_t *p, size_t count, cudaStream_t st) {
    k_g1a_from_g1p<<<grid_stride_blocks(count), 128, 0, st>>>(a, p, count);
}
void launch_bench_field(int field, int sqr, uint32_t *data, size_t count, int iters, cudaStream_t st) {
    if (field == 0) k_bench_field<FpDesc><<<blocks_for(count, 256), 256, 0, st>>>(data, count, iters, sqr);
    else k_bench_field<FrDesc><<<blocks_for(count, 256), 256, 0, st>>>(data, count, iters, sqr);
}
void launch_fingerprint(unsigned long long *out, const uint64_t *w, size_t n, cudaStream_t st) {
    k_fingerprint<<<148, 256, 0, st>>>(out, w, n);
}

}  // namespace fk
