// kernels_msm.cu -- fixed-base MSM of the FK20 pipeline.
//
// hext_fft[row][c] = sum_{i<16} tc_fft[row][i][c] * X_i[c]  (fk20_msm.cu:23-66;
// FK20Py/fk20_single.py:73-76).  The bases X_i[c] are fixed per setup, so each
// has a table of its signed-digit multiples: entry (w, e) = (e+1) 2^(cb w) X,
// e < 2^(cb-1), affine Montgomery (built by kernels_tables.cu).  A 255-bit
// scalar is recoded on the fly into ceil(255/cb) signed digits in
// [-2^(cb-1), 2^(cb-1)] and each nonzero digit costs one mixed addition of a
// gathered 96-byte entry: no doublings at all, against ~255 doublings + ~128
// additions per term in the reference's g1p_mul loop.  The accumulator is in
// XYZZ coordinates (x = X/ZZ, y = Y/ZZZ), whose mixed addition takes 8 M + 2 S
// (the complete projective one 11 M); its exceptional cases -- accumulator at
// infinity, equal or opposite points -- are tested and handled, so every sum
// is exact.  The result goes back to homogeneous projective coordinates.
// The Fp product and square out of line (one shared copy each): the mixed
// addition's ten inlined products overflowed the instruction cache.
#ifndef FK_MSM_OUTLINE
#define FK_MSM_OUTLINE 1
#endif
#if FK_MSM_OUTLINE
#define FK_FP_MUL_OUTLINE 1
#endif
#include <algorithm>

#include "../../include/fk20_b200.h"
#include "check.cuh"
#include "consts.cuh"
#include "launch.h"
#include "layout.cuh"

#ifndef FK_MSM_MINB
#define FK_MSM_MINB 1
#endif
// largest block size the launcher may use; the launch bounds cap registers
// at 65536 / (FK_MSM_MAX_THREADS * FK_MSM_MINB): 384 gives 168 registers, so
// three 128-thread blocks (12 warps) fit an SM (64-, 128- and 256-thread
// blocks launch as they are)
#ifndef FK_MSM_MAX_THREADS
#define FK_MSM_MAX_THREADS 384
#endif
constexpr int MSM_MAX_THREADS = FK_MSM_MAX_THREADS;

namespace fk {

cudaError_t upload_consts_msm() { return upload_module_consts(); }

FK_CHECK_WORD(msm)

// XYZZ point: x = X / ZZ, y = Y / ZZZ (ZZ^3 = ZZZ^2); ZZ = 0 is infinity
struct G1Z {
    Fp x, y, zz, zzz;
};
FK_D void g1z_set_inf(G1Z &a) {
    f_set_one(a.x);
    f_set_one(a.y);
    f_set_zero(a.zz);
    f_set_zero(a.zzz);
}
// a = 2 (qx, qy), affine q not infinity (y != 0 in the prime-order group):
// U = 2y, V = U^2, W = U V, S = x V, M = 3 x^2, X = M^2 - 2S,
// Y = M (S - X) - W y, ZZ = V, ZZZ = W
FK_D void g1z_dbl_affine(G1Z &a, const Fp &qx, const Fp &qy) {
    Fp u, v, w, sv, m, t;
    f_add(u, qy, qy);
    fp_sqr(v, u);
    fp_mul(w, u, v);
    fp_mul(sv, qx, v);
    fp_sqr(m, qx);
    f_add(t, m, m);
    f_add(m, t, m);
    fp_sqr(t, m);
    f_sub(t, t, sv);
    f_sub(a.x, t, sv);
    f_sub(t, sv, a.x);
    fp_mul(t, m, t);
    fp_mul(u, w, qy);
    f_sub(a.y, t, u);
    a.zz = v;
    a.zzz = w;
}
// a += (qx, qy), affine q not infinity (madd-2008-s: U2 = qx ZZ, S2 = qy ZZZ,
// P = U2 - X, R = S2 - Y, X3 = R^2 - P^3 - 2 X P^2, Y3 = R (X P^2 - X3) - Y P^3,
// ZZ3 = ZZ P^2, ZZZ3 = ZZZ P^3)
FK_D void g1z_madd(G1Z &a, const Fp &qx, const Fp &qy) {
    if (f_is_zero(a.zz)) {
        a.x = qx;
        a.y = qy;
        f_set_one(a.zz);
        f_set_one(a.zzz);
        return;
    }
    Fp u2, s2, p, r, pp, ppp, q, t;
    fp_mul(u2, qx, a.zz);
    fp_mul(s2, qy, a.zzz);
    f_sub(p, u2, a.x);
    f_sub(r, s2, a.y);
    if (f_is_zero(p)) {
        if (f_is_zero(r)) g1z_dbl_affine(a, qx, qy);  // a = q
        else g1z_set_inf(a);                          // a = -q
        return;
    }
    fp_sqr(pp, p);
    fp_mul(ppp, p, pp);
    fp_mul(q, a.x, pp);
    fp_sqr(t, r);
    f_sub(t, t, ppp);
    f_sub(t, t, q);
    f_sub(a.x, t, q);
    f_sub(t, q, a.x);
    fp_mul(t, r, t);
    fp_mul(s2, a.y, ppp);
    f_sub(a.y, t, s2);
    fp_mul(a.zz, a.zz, pp);
    fp_mul(a.zzz, a.zzz, ppp);
}
// homogeneous projective (X ZZZ, Y ZZ, ZZ ZZZ); infinity as (0, 1, 0)
FK_D void g1z_to_proj(G1P &r, const G1Z &a) {
    if (f_is_zero(a.zz)) {
        g1_set_inf(r);
        return;
    }
    fp_mul(r.x, a.x, a.zzz);
    fp_mul(r.y, a.y, a.zz);
    fp_mul(r.z, a.zz, a.zzz);
}

// acc += s * X for one base X, whose table `tb` holds (e+1) 2^(cb w) X for
// window w and e < 2^(cb-1): the 255-bit scalar s (9 words, s[8] = 0) is
// recoded into W signed digits in [-2^(cb-1), 2^(cb-1)] on the fly and every
// nonzero digit costs one mixed addition of a gathered 96-byte entry.
// Returns the recoding's final carry: nonzero when s needs more than W
// windows (the tables do not cover it).
FK_D int msm_add_scalar(G1Z &acc, const uint32_t s[9], const uint4 *__restrict__ tb, int W, int cb) {
    const int E = 1 << (cb - 1);
    const uint32_t mask = (1u << cb) - 1u;
    int carry = 0;
    for (int w = 0; w < W; w++) {
        const int bit = w * cb;
        const int wd = bit >> 5, sh = bit & 31;
        uint32_t raw = s[wd] >> sh;
        if (sh + cb > 32) raw |= s[wd + 1] << (32 - sh);
        int d = (int)(raw & mask) + carry;
        carry = d > E;
        if (carry) d -= (1 << cb);
        if (d != 0) {
            const int e = (d < 0 ? -d : d) - 1;
            const uint4 *ent = tb + ((size_t)w * E + e) * 6;
            Fp x, y;
            const uint4 q0 = ent[0], q1 = ent[1], q2 = ent[2], q3 = ent[3], q4 = ent[4], q5 = ent[5];
            x.w[0] = q0.x; x.w[1] = q0.y; x.w[2] = q0.z; x.w[3] = q0.w;
            x.w[4] = q1.x; x.w[5] = q1.y; x.w[6] = q1.z; x.w[7] = q1.w;
            x.w[8] = q2.x; x.w[9] = q2.y; x.w[10] = q2.z; x.w[11] = q2.w;
            y.w[0] = q3.x; y.w[1] = q3.y; y.w[2] = q3.z; y.w[3] = q3.w;
            y.w[4] = q4.x; y.w[5] = q4.y; y.w[6] = q4.z; y.w[7] = q4.w;
            y.w[8] = q5.x; y.w[9] = q5.y; y.w[10] = q5.z; y.w[11] = q5.w;
            // an entry (0, 0) encodes a base at infinity (not on the curve)
            if (!(f_is_zero(x) && f_is_zero(y))) {
                if (d < 0) f_neg(y, y);
                g1z_madd(acc, x, y);
            }
        }
    }
    return carry;
}

// One warp per (segment, column c, group g of 32 rows); lanes are rows.
// Warps are numbered segment by segment, g fastest, so the warps of a block
// read the same table column.
__global__ void __launch_bounds__(MSM_MAX_THREADS, FK_MSM_MINB) k_msm(const __grid_constant__ MsmArgs args) {
    const unsigned warp = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (warp >= args.warps) return;
    int k = 0;
    while (k + 1 < args.nseg && warp >= args.seg[k + 1].warp_start) k++;
    const MsmSeg &a = args.seg[k];
    const int m = 1 << a.log_m;
    const int lane = threadIdx.x & 31;
    const unsigned wl = warp - a.warp_start;
    const int g = (int)(wl % (unsigned)a.G), c = (int)(wl / (unsigned)a.G);
    if (!FK_CHECK(g_check_msm, k < args.nseg && c < m, FK20_CHECK_MSM_TILE)) return;
    if (args.test_check && warp == 0 && lane == 0) (void)FK_CHECK(g_check_msm, false, FK20_CHECK_MSM_PLANTED);
    const int row = g * 32 + lane;
    const bool live = row < a.rows;
    const int E = 1 << (a.cb - 1);
    // sum_i [s_i] X_i = phi(sum_i [s2_i] X_i) + sum_i [s1_i] X_i with
    // s_i = s1_i + s2_i lambda (the scalar tile holds s1 at uint4 0 and s2 at
    // uint4 1): the s2 halves first, then phi on the accumulator
    // ((X, Y, ZZ, ZZZ) -> (beta X, Y, ZZ, ZZZ)), then the s1 halves.
    G1Z accz;
    g1z_set_inf(accz);
#pragma unroll 1
    for (int half = 1; half >= 0; half--) {
#pragma unroll 1
        for (int i = 0; i < L_COLS; i++) {
            uint32_t s[9];
            const uint4 v = a.S[((((size_t)g * m + c) * L_COLS + i) * SCAL_Q + half) * 32 + lane];
            s[0] = v.x; s[1] = v.y; s[2] = v.z; s[3] = v.w;
#pragma unroll
            for (int k = 4; k < 9; k++) s[k] = 0;
            if (!live) {
#pragma unroll
                for (int k = 0; k < 4; k++) s[k] = 0;
            }
            const uint4 *tb = a.table + ((size_t)(i * m + c) * a.W) * E * 6;
            const int carry = msm_add_scalar(accz, s, tb, a.W, a.cb);
            (void)FK_CHECK(g_check_msm, carry == 0, FK20_CHECK_MSM_CARRY);
        }
        if (half) {
            Fp beta;
#pragma unroll
            for (int k = 0; k < 12; k++) beta.w[k] = beta_mont(k);
            fp_mul(accz.x, accz.x, beta);
        }
    }
    G1P acc;
    g1z_to_proj(acc, accz);
    if (args.times_m) {
        for (int t = 0; t < a.log_m; t++) g1_dbl(acc, acc);
    }
    tile_store(a.D + tile_index(g, m, c), lane, acc);
}

// ---------------------------------------------------------------- KZG commitments
// commitment[row] = sum_i poly[row][i] * s_i over fixed-base tables of the
// setup points s_i (commit_to_poly, FK20Py/kzg_proofs.py:159-163).  Pass 1:
// warp (g, p) sums bases [p n / P, (p+1) n / P) for the 32 rows of group g
// into a partial-sum tile, P = commit_parts(rows, n) warps per group, chosen
// so that pass 1 is one wave of resident warps (whole warps of fixed chunks
// left a second, mostly idle wave); pass 2: one thread per row adds its P
// partials.
__global__ void __launch_bounds__(128) k_commit_partial(uint4 *__restrict__ part, const uint64_t *__restrict__ poly,
                                                        const uint4 *__restrict__ table, int rows, int n, int W,
                                                        int cb, int P) {
    const int G = (rows + 31) / 32;
    const unsigned warp = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (warp >= (unsigned)G * P) return;
    const int lane = threadIdx.x & 31;
    const int g = (int)(warp % (unsigned)G), c = (int)(warp / (unsigned)G);
    const int row = g * 32 + lane;
    const bool live = row < rows;
    const int E = 1 << (cb - 1);
    const int i0 = (int)((long long)c * n / P), i1 = (int)((long long)(c + 1) * n / P);
    G1Z accz;
    g1z_set_inf(accz);
    for (int i = i0; i < i1; i++) {
        uint32_t s[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        if (live) {
            Fr f;
            fr_from_ref(f, poly + 4 * ((size_t)row * n + i));
#pragma unroll
            for (int k = 0; k < 8; k++) s[k] = f.w[k];
        }
        (void)msm_add_scalar(accz, s, table + (size_t)i * W * E * 6, W, cb);
    }
    G1P acc;
    g1z_to_proj(acc, accz);
    tile_store(part + tile_index(g, P, c), lane, acc);
}

__global__ void k_commit_reduce(uint64_t *__restrict__ out, const uint4 *__restrict__ part, int rows, int P) {
    for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < rows; row += gridDim.x * blockDim.x) {
        const int g = row >> 5, lane = row & 31;
        G1P acc, q;
        tile_load(acc, part + tile_index(g, P, 0), lane);
        for (int c = 1; c < P; c++) {
            tile_load(q, part + tile_index(g, P, c), lane);
            g1_add(acc, acc, q);
        }
        g1p_to_ref(out + 18 * (size_t)row, acc);
    }
}

// pass-1 warps per group of 32 rows: one wave of the warps the device holds
// at once, at least one, at most one per base
int commit_parts(int rows, int n) {
    static int resident = 0;  // warps of k_commit_partial resident on the device
    if (!resident) {
        int dev = 0, sms = 1, bps = 1;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_commit_partial, 128, 0) != cudaSuccess || bps < 1) {
            cudaGetLastError();
            bps = 1;
        }
        resident = sms * bps * 4;
    }
    const int G = (rows + 31) / 32;
    return std::max(1, std::min(n, resident / G));
}

void launch_commit(uint64_t *out, uint4 *part, const uint64_t *poly, const uint4 *table, int rows, int n, int W,
                   int cb, cudaStream_t st) {
    const int P = commit_parts(rows, n);
    const unsigned warps = (unsigned)((rows + 31) / 32) * (unsigned)P;
    k_commit_partial<<<blocks_for(warps, 4), 128, 0, st>>>(part, poly, table, rows, n, W, cb, P);
    k_commit_reduce<<<blocks_for((size_t)rows, 128), 128, 0, st>>>(out, part, rows, P);
}

void launch_msm(const MsmArgs &a, int threads, cudaStream_t st) {
    if (threads != 64 && threads != 128 && threads != 256) threads = 128;
    if (threads > MSM_MAX_THREADS) threads = MSM_MAX_THREADS;
    k_msm<<<blocks_for(a.warps, (unsigned)threads / 32), threads, 0, st>>>(a);
}

}  // namespace fk
