// layout.cuh -- HBM layouts of the engine.
//
// Reference layouts (the ABI): fr_t = 4 x u64, g1p_t = {x,y,z} 18 x u64, all
// standard form, array-of-structures, row-major ([row][k] as in
// fk20_poly2h_fft.cu:40-46).
//
// Engine layouts ("row-interleaved"): rows are processed 32 at a time, one
// row per lane of a warp, and every warp of a G1 FFT stage or MSM column works
// on the SAME butterfly / column of 32 different rows.  Fixed-scalar programs
// are therefore warp-uniform, and every load is a coalesced 512-byte uint4
// sweep:
//   point tile  D[g][i][q][lane]  uint4, q = 0..8 holds words 4q..4q+3 of the
//                                 36-word projective Montgomery point (x: 0-11,
//                                 y: 12-23, z: 24-35); g = row/32, lane = row%32
//   scalar tile S[g][c][t][q][lane] uint4, q = 0..1 holds words of the 8-word
//                                 standard-form Fr scalar t of column c
// Fixed-base table entry (b, w, e): 6 uint4 (affine x, y Montgomery) at
//   ((b * W + w) * E + e) * 6.
#pragma once
#include "g1.cuh"

namespace fk {

constexpr int TILE_Q = 9;  // uint4 per projective point
constexpr int SCAL_Q = 2;  // uint4 per Fr scalar

FK_D size_t tile_index(int g, int m, int i) { return ((size_t)g * m + i) * TILE_Q * 32; }

FK_D void tile_load(G1P &p, const uint4 *__restrict__ base, int lane) {
    uint32_t w[36];
#pragma unroll
    for (int q = 0; q < TILE_Q; q++) {
        uint4 v = base[q * 32 + lane];
        w[4 * q] = v.x; w[4 * q + 1] = v.y; w[4 * q + 2] = v.z; w[4 * q + 3] = v.w;
    }
#pragma unroll
    for (int k = 0; k < 12; k++) { p.x.w[k] = w[k]; p.y.w[k] = w[12 + k]; p.z.w[k] = w[24 + k]; }
}

FK_D void tile_store(uint4 *__restrict__ base, int lane, const G1P &p) {
    uint32_t w[36];
#pragma unroll
    for (int k = 0; k < 12; k++) { w[k] = p.x.w[k]; w[12 + k] = p.y.w[k]; w[24 + k] = p.z.w[k]; }
#pragma unroll
    for (int q = 0; q < TILE_Q; q++) base[q * 32 + lane] = make_uint4(w[4 * q], w[4 * q + 1], w[4 * q + 2], w[4 * q + 3]);
}

// tile point -> strided slot (shared memory), one uint4 at a time, without
// holding the whole point in registers
FK_D void tile_to_slot(const StridedPoint &slot, const uint4 *__restrict__ base, int lane) {
#pragma unroll
    for (int q = 0; q < TILE_Q; q++) {
        const uint4 v = base[q * 32 + lane];
        slot.base[(4 * q) * slot.stride] = v.x;
        slot.base[(4 * q + 1) * slot.stride] = v.y;
        slot.base[(4 * q + 2) * slot.stride] = v.z;
        slot.base[(4 * q + 3) * slot.stride] = v.w;
    }
}

// reference g1p_t (18 x u64 standard form, any representative) -> Montgomery point.
// Any (X, Y, 0) is the point at infinity (reference G1P_ANYINF, g1.cuh:14).
FK_D void g1p_from_ref(G1P &p, const uint64_t *__restrict__ g) {
    Fp t;
#pragma unroll
    for (int k = 0; k < 6; k++) { t.w[2 * k] = (uint32_t)g[k]; t.w[2 * k + 1] = (uint32_t)(g[k] >> 32); }
    f_to_mont(p.x, t);
#pragma unroll
    for (int k = 0; k < 6; k++) { t.w[2 * k] = (uint32_t)g[6 + k]; t.w[2 * k + 1] = (uint32_t)(g[6 + k] >> 32); }
    f_to_mont(p.y, t);
#pragma unroll
    for (int k = 0; k < 6; k++) { t.w[2 * k] = (uint32_t)g[12 + k]; t.w[2 * k + 1] = (uint32_t)(g[12 + k] >> 32); }
    f_to_mont(p.z, t);
    if (f_is_zero(p.z)) g1_set_inf(p);
}

// Montgomery point -> reference g1p_t, canonical limbs; infinity as (0, 1, 0)
FK_D void g1p_to_ref(uint64_t *__restrict__ g, const G1P &p) {
    Fp t;
    if (f_is_zero(p.z)) {
#pragma unroll
        for (int k = 0; k < 18; k++) g[k] = 0;
        g[6] = 1;
        return;
    }
    f_from_mont(t, p.x);
#pragma unroll
    for (int k = 0; k < 6; k++) g[k] = (uint64_t)t.w[2 * k] | ((uint64_t)t.w[2 * k + 1] << 32);
    f_from_mont(t, p.y);
#pragma unroll
    for (int k = 0; k < 6; k++) g[6 + k] = (uint64_t)t.w[2 * k] | ((uint64_t)t.w[2 * k + 1] << 32);
    f_from_mont(t, p.z);
#pragma unroll
    for (int k = 0; k < 6; k++) g[12 + k] = (uint64_t)t.w[2 * k] | ((uint64_t)t.w[2 * k + 1] << 32);
}

// reference fr_t (any 256-bit representative) -> canonical standard-form Fr
FK_D void fr_from_ref(Fr &s, const uint64_t *__restrict__ x) {
    uint32_t t[8];
#pragma unroll
    for (int k = 0; k < 4; k++) { t[2 * k] = (uint32_t)x[k]; t[2 * k + 1] = (uint32_t)(x[k] >> 32); }
    // x < 2^256 < 3r: at most two subtractions of r
    f_reduce_once<FrDesc>(t, t);
    f_reduce_once<FrDesc>(s.w, t);
}

FK_D void fr_to_ref(uint64_t *__restrict__ x, const Fr &s) {
#pragma unroll
    for (int k = 0; k < 4; k++) x[k] = (uint64_t)s.w[2 * k] | ((uint64_t)s.w[2 * k + 1] << 32);
}

FK_HD unsigned bitrev(unsigned v, int bits) {
#if defined(__CUDA_ARCH__)
    return __brev(v) >> (32 - bits);
#else
    unsigned r = 0;
    for (int i = 0; i < bits; i++) r |= ((v >> i) & 1u) << (bits - 1 - i);
    return r;
#endif
}

}  // namespace fk
