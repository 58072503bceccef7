// kernels_tables.cu -- fixed-base tables for the MSM (setup time).
//
// For each base X_b (b = i*m + c of xext_fft) and window w the table holds
// (e+1) 2^(cb w) X'_b for e < 2^(cb-1), affine Montgomery, X'_b = X_b / m
// (the inverse FFT's 1/m folded into the bases, fk20_single.py:78-84).
// Replaces the reference's comb tables (fk20_msm_makelut, fk20_msm.cu:79-141,
// one thread per base).  Three passes over a slab of bases:
//   k_table_windows : X'_b and its window multiples 2^(cb w) X'_b
//   k_table_fill    : (e+1) * window base for a chunk of TAB_CHUNK entries;
//                     X, Y into the table slot, Z into a scratch array
//   k_table_affine  : batch inversion over the chunk (Montgomery's trick),
//                     then (X/Z, Y/Z) into the slot; infinity as (0, 0)
#include "consts.cuh"
#include "launch.h"
#include "layout.cuh"

namespace fk {

cudaError_t upload_consts_tables() { return upload_module_consts(); }
size_t table_window_base_bytes() { return sizeof(G1P); }
size_t table_z_bytes() { return sizeof(Fp); }

__global__ void k_table_windows(G1P *__restrict__ wb, const uint64_t *__restrict__ xext, int b0, int nb, int W, int cb,
                                int prog_scale) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nb) return;
    G1P p;
    g1p_from_ref(p, xext + 18 * (size_t)(b0 + t));
    if (prog_scale >= 0) g1_mul_prog(p, p, c_prog[prog_scale]);
    for (int w = 0; w < W; w++) {
        wb[(size_t)t * W + w] = p;
        for (int k = 0; k < cb; k++) g1_dbl(p, p);
    }
}

__device__ void store_xy(uint4 *ent, const Fp &x, const Fp &y) {
    ent[0] = make_uint4(x.w[0], x.w[1], x.w[2], x.w[3]);
    ent[1] = make_uint4(x.w[4], x.w[5], x.w[6], x.w[7]);
    ent[2] = make_uint4(x.w[8], x.w[9], x.w[10], x.w[11]);
    ent[3] = make_uint4(y.w[0], y.w[1], y.w[2], y.w[3]);
    ent[4] = make_uint4(y.w[4], y.w[5], y.w[6], y.w[7]);
    ent[5] = make_uint4(y.w[8], y.w[9], y.w[10], y.w[11]);
}

__device__ void load_xy(const uint4 *ent, Fp &x, Fp &y) {
    const uint4 q0 = ent[0], q1 = ent[1], q2 = ent[2], q3 = ent[3], q4 = ent[4], q5 = ent[5];
    x.w[0] = q0.x; x.w[1] = q0.y; x.w[2] = q0.z; x.w[3] = q0.w;
    x.w[4] = q1.x; x.w[5] = q1.y; x.w[6] = q1.z; x.w[7] = q1.w;
    x.w[8] = q2.x; x.w[9] = q2.y; x.w[10] = q2.z; x.w[11] = q2.w;
    y.w[0] = q3.x; y.w[1] = q3.y; y.w[2] = q3.z; y.w[3] = q3.w;
    y.w[4] = q4.x; y.w[5] = q4.y; y.w[6] = q4.z; y.w[7] = q4.w;
    y.w[8] = q5.x; y.w[9] = q5.y; y.w[10] = q5.z; y.w[11] = q5.w;
}

__global__ void k_table_fill(uint4 *__restrict__ table, Fp *__restrict__ zs, const G1P *__restrict__ wb, int b0, int nb,
                             int W, int cb) {
    const int E = 1 << (cb - 1);
    const int chunks = E / TAB_CHUNK;
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (t >= (size_t)nb * W * chunks) return;
    const int ch = (int)(t % chunks);
    const size_t bw = t / chunks;  // (base - b0) * W + w
    const G1P base = wb[bw];
    const int e0 = ch * TAB_CHUNK + 1;
    G1P acc;
    g1_set_inf(acc);
    for (int bit = 31 - __clz(e0); bit >= 0; bit--) {
        g1_dbl(acc, acc);
        if ((e0 >> bit) & 1) g1_add(acc, acc, base);
    }
    const size_t slot0 = ((size_t)b0 * W + bw) * E + (size_t)ch * TAB_CHUNK;
    for (int k = 0; k < TAB_CHUNK; k++) {
        store_xy(table + (slot0 + k) * 6, acc.x, acc.y);
        zs[t * TAB_CHUNK + k] = acc.z;
        g1_add(acc, acc, base);
    }
}

__global__ void k_table_affine(uint4 *__restrict__ table, const Fp *__restrict__ zs, int b0, int nb, int W, int cb) {
    const int E = 1 << (cb - 1);
    const int chunks = E / TAB_CHUNK;
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (t >= (size_t)nb * W * chunks) return;
    const int ch = (int)(t % chunks);
    const size_t bw = t / chunks;
    const size_t slot0 = ((size_t)b0 * W + bw) * E + (size_t)ch * TAB_CHUNK;
    Fp pre[TAB_CHUNK];
    Fp acc;
    f_set_one(acc);
    for (int k = 0; k < TAB_CHUNK; k++) {
        pre[k] = acc;
        const Fp z = zs[t * TAB_CHUNK + k];
        if (!f_is_zero(z)) f_mul(acc, acc, z);
    }
    Fp inv;
    f_inv(inv, acc);
    for (int k = TAB_CHUNK - 1; k >= 0; k--) {
        const Fp z = zs[t * TAB_CHUNK + k];
        uint4 *ent = table + (slot0 + k) * 6;
        Fp x, y;
        if (f_is_zero(z)) {
            f_set_zero(x);
            f_set_zero(y);
        } else {
            Fp zi, X, Y;
            f_mul(zi, inv, pre[k]);
            f_mul(inv, inv, z);
            load_xy(ent, X, Y);
            f_mul(x, X, zi);
            f_mul(y, Y, zi);
        }
        store_xy(ent, x, y);
    }
}

void launch_table_windows(void *wb, const uint64_t *xext, int b0, int nb, int W, int cb, int prog_scale,
                          cudaStream_t st) {
    k_table_windows<<<blocks_for(nb, 64), 64, 0, st>>>((G1P *)wb, xext, b0, nb, W, cb, prog_scale);
}
void launch_table_fill(uint4 *table, void *zs, const void *wb, int b0, int nb, int W, int cb, cudaStream_t st) {
    const size_t n = (size_t)nb * W * ((1 << (cb - 1)) / TAB_CHUNK);
    k_table_fill<<<blocks_for(n, 128), 128, 0, st>>>(table, (Fp *)zs, (const G1P *)wb, b0, nb, W, cb);
}
void launch_table_affine(uint4 *table, const void *zs, int b0, int nb, int W, int cb, cudaStream_t st) {
    const size_t n = (size_t)nb * W * ((1 << (cb - 1)) / TAB_CHUNK);
    k_table_affine<<<blocks_for(n, 128), 128, 0, st>>>(table, (const Fp *)zs, b0, nb, W, cb);
}

}  // namespace fk
