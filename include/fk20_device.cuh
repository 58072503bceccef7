/*
 * fk20_device.cuh -- the reference's fp_* / fr_* / g1p_* DEVICE API as a
 * header-only library (fp.cuh:16-41, fr.cuh:33-58, g1.cuh:31-96 of
 * lCardosoSantos/FK20-CUDA): same names, same signatures, same value
 * conventions, for CUDA code that calls these functions from its own kernels.
 *
 *  - fp_t / fr_t / g1p_t / g1a_t are the reference layouts (include/fk20_b200.h):
 *    standard (non-Montgomery) little-endian 64-bit words; inputs may be any
 *    384-bit (fp_t) or 256-bit (fr_t) representative; results are canonical.
 *  - g1p_t is homogeneous projective (x = X/Z, y = Y/Z); any (0, y != 0, 0)
 *    is the point at infinity (G1P_ANYINF), written as (0, 1, 0).
 *
 * Cost model.  Words are only reduced on the way in (conditional subtractions
 * of 8p, 4p, 2p, p -- or 2r, r -- so any 384-/256-bit representative is
 * accepted) and the engine's Montgomery arithmetic runs on the standard-form
 * words directly:
 *  - additions, subtractions, negation, x2..x12, comparisons: no products;
 *  - fp_mul / fr_mul / squares: MontMul(x, y) = x y R^-1, then one more
 *    Montgomery product by R^2 mod p restores x y -- two products where a
 *    convert-in / multiply / convert-out wrapper needs four;
 *  - G1: homogeneous projective coordinates are defined up to a common
 *    non-zero factor, and standard-form words (X, Y, Z) read as Montgomery
 *    values are (X, Y, Z) R^-1 -- the same point.  The engine's complete
 *    formulas (whose only constant, b3 = 12, is applied by additions) therefore
 *    run on the words as they are, with no conversion.  A g1p_t result is the
 *    reference's point, but its coordinates may differ from the reference's by
 *    a common factor (a power of R): compare with g1p_eq, or normalise with
 *    g1a_fromG1p, as the reference's own tests do (g1p_compare.cu:23).
 * The batched host entry points and the FK20 pipeline keep values in
 * Montgomery form throughout.  The block-level fr_fft / fr_ift / g1p_fft /
 * g1p_ift device functions of the reference are provided as host launchers
 * in fk20_b200.h instead.
 *
 * Use: nvcc -gencode arch=compute_100a,code=sm_100a -I include ... with this
 * repository's layout (the header includes ../fk20-cuda_b200/csrc/).
 */
#ifndef FK20_DEVICE_CUH
#define FK20_DEVICE_CUH

#include <stdio.h>

#include "fk20_b200.h"
#include "../fk20-cuda_b200/csrc/g1.cuh"

#define G1P_ANYINF 1

namespace fk20_device_detail {
using namespace fk;

template <class F, int W>
__device__ __forceinline__ void load_words(Elem<F> &e, const uint64_t (&x)[W]) {
#pragma unroll
    for (int k = 0; k < W; k++) { e.w[2 * k] = (uint32_t)x[k]; e.w[2 * k + 1] = (uint32_t)(x[k] >> 32); }
}
template <class F, int W>
__device__ __forceinline__ void store_words(uint64_t (&x)[W], const Elem<F> &e) {
#pragma unroll
    for (int k = 0; k < W; k++) x[k] = (uint64_t)e.w[2 * k] | ((uint64_t)e.w[2 * k + 1] << 32);
}
// e mod m for any e < 2^(32N): subtract 2^k m where it fits, k = K..0.  Fp:
// 2^384 < 10 p, so K = 3 (8p < 2^384); Fr: 2^256 < 3 r, so K = 1.
template <class F, int K>
__device__ __forceinline__ void reduce_any(Elem<F> &e) {
#pragma unroll
    for (int k = K; k >= 0; k--) {
        uint32_t m[F::N], t[F::N];
#pragma unroll
        for (int i = 0; i < F::N; i++) m[i] = (F::mod(i) << k) | (i > 0 && k > 0 ? F::mod(i - 1) >> (32 - k) : 0u);
        const uint32_t borrow = ch_sub<F>(t, e.w, m);  // all ones when e < 2^k m
#pragma unroll
        for (int i = 0; i < F::N; i++) e.w[i] = (e.w[i] & borrow) | (t[i] & ~borrow);
    }
}
// any standard-form representative -> canonical standard form (no products)
__device__ __forceinline__ void canon(Fp &e, const fp_t &x) { load_words(e, x); reduce_any<FpDesc, 3>(e); }
__device__ __forceinline__ void canon(Fr &e, const fr_t &x) { load_words(e, x); reduce_any<FrDesc, 1>(e); }
// standard-form product of canonical a, b: MontMul(R^2, MontMul(a, b)) = a b
template <class F>
__device__ __forceinline__ void std_mul(Elem<F> &r, const Elem<F> &a, const Elem<F> &b) {
    Elem<F> t;
    f_mul(t, a, b);
    f_to_mont(r, t);
}
template <class F>
__device__ __forceinline__ void std_sqr(Elem<F> &r, const Elem<F> &a) {
    Elem<F> t;
    f_sqr(t, a);
    f_to_mont(r, t);
}
// standard-form inverse of canonical a: f_inv reads a as the Montgomery form
// of a R^-1 and returns the words of a^-1 R^2; two Montgomery products by 1
// take off R^2 (inv(0) = 0)
template <class F>
__device__ __forceinline__ void std_inv(Elem<F> &r, const Elem<F> &a) {
    Elem<F> t;
    f_inv(t, a);
    f_from_mont(t, t);
    f_from_mont(r, t);
}
// Montgomery form -> canonical standard form
__device__ __forceinline__ void plain(fp_t &z, const Fp &m) { Fp t; f_from_mont(t, m); store_words(z, t); }

// a g1p_t as engine coordinates: canonical words, no conversion (the same
// projective point, see the header comment); any (0, y != 0, 0) -> infinity
__device__ __forceinline__ void point(G1P &p, const g1p_t &q) {
    canon(p.x, q.x);
    canon(p.y, q.y);
    canon(p.z, q.z);
    if (f_is_zero(p.z)) g1_set_inf(p);
}
__device__ __forceinline__ void unpoint(g1p_t &q, const G1P &p) {
    if (f_is_zero(p.z)) {
#pragma unroll
        for (int k = 0; k < 6; k++) q.x[k] = q.y[k] = q.z[k] = 0;
        q.y[0] = 1;
        return;
    }
    store_words(q.x, p.x);
    store_words(q.y, p.y);
    store_words(q.z, p.z);
}
// affine (x, y) -> (x : y : 1) with Z the standard-form word 1 (the Montgomery
// one would give the point (x R^-1 : y R^-1 : 1), another point); (0, 0) is
// the point at infinity
__device__ __forceinline__ void point(G1P &p, const g1a_t &a) {
    canon(p.x, a.x);
    canon(p.y, a.y);
    f_set_zero(p.z);
    p.z.w[0] = 1;
    if (f_is_zero(p.x) && f_is_zero(p.y)) g1_set_inf(p);
}
}  // namespace fk20_device_detail

// ------------------------------------------------------------------ Fp (fp.cuh:16-41)
__device__ __host__ inline void fp_fromUint64(fp_t &z, const uint64_t *x) { for (int k = 0; k < 6; k++) z[k] = x[k]; }
__device__ inline void fp_toUint64(uint64_t *z, const fp_t &x) { for (int k = 0; k < 6; k++) z[k] = x[k]; }
__device__ __host__ inline void fp_cpy(fp_t &z, const fp_t &x) { for (int k = 0; k < 6; k++) z[k] = x[k]; }
__device__ __host__ inline void fp_zero(fp_t &z) { for (int k = 0; k < 6; k++) z[k] = 0; }
__device__ __host__ inline void fp_one(fp_t &z) { fp_zero(z); z[0] = 1; }

#define FK20_DEV_FP_UNARY(name, body)                         \
    __device__ inline void name(fp_t &z, const fp_t &x) {     \
        using namespace fk20_device_detail;                   \
        fk::Fp a, r;                                          \
        canon(a, x);                                          \
        body;                                                 \
        store_words(z, r);                                    \
    }
FK20_DEV_FP_UNARY(fp_neg, fk::f_neg(r, a))
FK20_DEV_FP_UNARY(fp_x2, fk::f_add(r, a, a))
FK20_DEV_FP_UNARY(fp_x3, { fk::f_add(r, a, a); fk::f_add(r, r, a); })
FK20_DEV_FP_UNARY(fp_x4, { fk::f_add(r, a, a); fk::f_add(r, r, r); })
FK20_DEV_FP_UNARY(fp_x8, { fk::f_add(r, a, a); fk::f_add(r, r, r); fk::f_add(r, r, r); })
FK20_DEV_FP_UNARY(fp_x12, fk::f_mul12(r, a))
FK20_DEV_FP_UNARY(fp_sqr, std_sqr(r, a))
FK20_DEV_FP_UNARY(fp_inv, std_inv(r, a))
#undef FK20_DEV_FP_UNARY

__device__ inline void fp_reduce6(fp_t &z) {
    using namespace fk20_device_detail;
    fk::Fp a;
    canon(a, z);
    store_words(z, a);
}
__device__ inline void fp_add(fp_t &z, const fp_t &x, const fp_t &y) {
    using namespace fk20_device_detail;
    fk::Fp a, b;
    canon(a, x);
    canon(b, y);
    fk::f_add(a, a, b);
    store_words(z, a);
}
__device__ inline void fp_sub(fp_t &z, const fp_t &x, const fp_t &y) {
    using namespace fk20_device_detail;
    fk::Fp a, b;
    canon(a, x);
    canon(b, y);
    fk::f_sub(a, a, b);
    store_words(z, a);
}
__device__ inline void fp_mul(fp_t &z, const fp_t &x, const fp_t &y) {
    using namespace fk20_device_detail;
    fk::Fp a, b;
    canon(a, x);
    canon(b, y);
    std_mul(a, a, b);
    store_words(z, a);
}
// z = v w + x y (fp_mma.cu:21): MontMul(v, w) + MontMul(x, y) = (v w + x y) R^-1,
// then one product by R^2 -- three products
__device__ inline void fp_mma(fp_t &z, const fp_t &v, const fp_t &w, const fp_t &x, const fp_t &y) {
    using namespace fk20_device_detail;
    fk::Fp a, b, c, d;
    canon(a, v);
    canon(b, w);
    canon(c, x);
    canon(d, y);
    fk::f_mul(a, a, b);
    fk::f_mul(c, c, d);
    fk::f_add(a, a, c);
    fk::f_to_mont(a, a);
    store_words(z, a);
}
__device__ inline bool fp_eq(const fp_t &x, const fp_t &y) {
    using namespace fk20_device_detail;
    fk::Fp a, b;
    canon(a, x);
    canon(b, y);
    return fk::f_eq(a, b);
}
__device__ inline bool fp_neq(const fp_t &x, const fp_t &y) { return !fp_eq(x, y); }
__device__ inline bool fp_iszero(const fp_t &x) {
    using namespace fk20_device_detail;
    fk::Fp a;
    canon(a, x);
    return fk::f_is_zero(a);
}
__device__ inline bool fp_nonzero(const fp_t &x) { return !fp_iszero(x); }
__device__ inline bool fp_isone(const fp_t &x) {
    fp_t o;
    fp_one(o);
    return fp_eq(x, o);
}
__device__ inline void fp_print(const char *s, const fp_t &x) {
    printf("%s%016llx%016llx%016llx%016llx%016llx%016llx\n", s, (unsigned long long)x[5], (unsigned long long)x[4],
           (unsigned long long)x[3], (unsigned long long)x[2], (unsigned long long)x[1], (unsigned long long)x[0]);
}

// ------------------------------------------------------------------ Fr (fr.cuh:33-58; in-place forms)
__device__ __host__ inline void fr_fromUint64(fr_t &z, const uint64_t *x) { for (int k = 0; k < 4; k++) z[k] = x[k]; }
__device__ inline void fr_toUint64(const fr_t &x, uint64_t *z) { for (int k = 0; k < 4; k++) z[k] = x[k]; }
__device__ __host__ inline void fr_cpy(fr_t &z, const fr_t &x) { for (int k = 0; k < 4; k++) z[k] = x[k]; }
__device__ __host__ inline void fr_zero(fr_t &z) { for (int k = 0; k < 4; k++) z[k] = 0; }
__device__ __host__ inline void fr_one(fr_t &z) { fr_zero(z); z[0] = 1; }

#define FK20_DEV_FR_INPLACE(name, body)                       \
    __device__ inline void name(fr_t &z) {                    \
        using namespace fk20_device_detail;                   \
        fk::Fr a, r;                                          \
        canon(a, z);                                          \
        body;                                                 \
        store_words(z, r);                                    \
    }
FK20_DEV_FR_INPLACE(fr_reduce4, r = a)
FK20_DEV_FR_INPLACE(fr_neg, fk::f_neg(r, a))
FK20_DEV_FR_INPLACE(fr_x2, fk::f_add(r, a, a))
FK20_DEV_FR_INPLACE(fr_x3, { fk::f_add(r, a, a); fk::f_add(r, r, a); })
FK20_DEV_FR_INPLACE(fr_x4, { fk::f_add(r, a, a); fk::f_add(r, r, r); })
FK20_DEV_FR_INPLACE(fr_x8, { fk::f_add(r, a, a); fk::f_add(r, r, r); fk::f_add(r, r, r); })
FK20_DEV_FR_INPLACE(fr_x12, fk::f_mul12(r, a))
FK20_DEV_FR_INPLACE(fr_sqr, std_sqr(r, a))
FK20_DEV_FR_INPLACE(fr_inv, std_inv(r, a))
#undef FK20_DEV_FR_INPLACE

#define FK20_DEV_FR_BINARY(name, op)                          \
    __device__ inline void name(fr_t &z, const fr_t &x) {     \
        using namespace fk20_device_detail;                   \
        fk::Fr a, b;                                          \
        canon(a, z);                                          \
        canon(b, x);                                          \
        op(a, a, b);                                          \
        store_words(z, a);                                    \
    }
FK20_DEV_FR_BINARY(fr_add, fk::f_add)
FK20_DEV_FR_BINARY(fr_sub, fk::f_sub)
FK20_DEV_FR_BINARY(fr_mul, std_mul)
#undef FK20_DEV_FR_BINARY

// (x, y) <- (x + y, x - y)   (fr_addsub.cu:18)
__device__ inline void fr_addsub(fr_t &x, fr_t &y) {
    using namespace fk20_device_detail;
    fk::Fr a, b, s, d;
    canon(a, x);
    canon(b, y);
    fk::f_add(s, a, b);
    fk::f_sub(d, a, b);
    store_words(x, s);
    store_words(y, d);
}
__device__ inline bool fr_eq(const fr_t &x, const fr_t &y) {
    using namespace fk20_device_detail;
    fk::Fr a, b;
    canon(a, x);
    canon(b, y);
    return fk::f_eq(a, b);
}
__device__ inline bool fr_neq(const fr_t &x, const fr_t &y) { return !fr_eq(x, y); }
__device__ inline bool fr_iszero(const fr_t &x) {
    using namespace fk20_device_detail;
    fk::Fr a;
    canon(a, x);
    return fk::f_is_zero(a);
}
__device__ inline bool fr_nonzero(const fr_t &x) { return !fr_iszero(x); }
__device__ inline bool fr_isone(const fr_t &x) {
    fr_t o;
    fr_one(o);
    return fr_eq(x, o);
}
__device__ inline void fr_print(const char *s, const fr_t &x) {
    printf("%s%016llx%016llx%016llx%016llx\n", s, (unsigned long long)x[3], (unsigned long long)x[2],
           (unsigned long long)x[1], (unsigned long long)x[0]);
}

// ------------------------------------------------------------------ G1 (g1.cuh:31-96; in-place forms)
__device__ __host__ inline void g1p_inf(g1p_t &p) {
    for (int k = 0; k < 6; k++) p.x[k] = p.y[k] = p.z[k] = 0;
    p.y[0] = 1;
}
__device__ __host__ inline void g1a_inf(g1a_t &a) {
    for (int k = 0; k < 6; k++) a.x[k] = a.y[k] = 0;
}
// the standard generator (x, y, 1)
__device__ __host__ inline void g1a_gen(g1a_t &a) {
    const uint64_t x[6] = {0xFB3AF00ADB22C6BBull, 0x6C55E83FF97A1AEFull, 0xA14E3A3F171BAC58ull,
                           0xC3688C4F9774B905ull, 0x2695638C4FA9AC0Full, 0x17F1D3A73197D794ull};
    const uint64_t y[6] = {0x0CAA232946C5E7E1ull, 0xD03CC744A2888AE4ull, 0x00DB18CB2C04B3EDull,
                           0xFCF5E095D5D00AF6ull, 0xA09E30ED741D8AE4ull, 0x08B3F481E3AAA0F1ull};
    for (int k = 0; k < 6; k++) a.x[k] = x[k], a.y[k] = y[k];
}
__device__ __host__ inline void g1p_gen(g1p_t &p) {
    g1a_t a;
    g1a_gen(a);
    for (int k = 0; k < 6; k++) p.x[k] = a.x[k], p.y[k] = a.y[k], p.z[k] = 0;
    p.z[0] = 1;
}
__device__ __host__ inline void g1p_cpy(g1p_t &p, const g1p_t &q) {
    for (int k = 0; k < 6; k++) p.x[k] = q.x[k], p.y[k] = q.y[k], p.z[k] = q.z[k];
}
__device__ __host__ inline void g1a_cpy(g1a_t &a, const g1a_t &b) {
    for (int k = 0; k < 6; k++) a.x[k] = b.x[k], a.y[k] = b.y[k];
}
__device__ __host__ inline void g1p_fromUint64(g1p_t &p, const uint64_t *x, const uint64_t *y, const uint64_t *z) {
    for (int k = 0; k < 6; k++) p.x[k] = x[k], p.y[k] = y[k], p.z[k] = z[k];
}
__device__ inline void g1p_toUint64(const g1p_t &p, uint64_t *x, uint64_t *y, uint64_t *z) {
    for (int k = 0; k < 6; k++) x[k] = p.x[k], y[k] = p.y[k], z[k] = p.z[k];
}
__device__ __host__ inline void g1a_fromUint64(g1a_t &a, const uint64_t *x, const uint64_t *y) {
    for (int k = 0; k < 6; k++) a.x[k] = x[k], a.y[k] = y[k];
}
__device__ __host__ inline void g1a_fromFp(g1a_t &a, const fp_t &x, const fp_t &y) {
    for (int k = 0; k < 6; k++) a.x[k] = x[k], a.y[k] = y[k];
}
__device__ inline void g1p_fromG1a(g1p_t &p, const g1a_t &a) {
    using namespace fk20_device_detail;
    fk::G1P q;
    point(q, a);
    unpoint(p, q);
}
// affine (x, y); infinity -> (0, 0)   (g1p.cu:168)
__device__ inline void g1a_fromG1p(g1a_t &a, const g1p_t &p) {
    using namespace fk20_device_detail;
    fk::G1P q;
    point(q, p);
    if (fk::f_is_zero(q.z)) {
        g1a_inf(a);
        return;
    }
    fk::g1_normalize(q);
    plain(a.x, q.x);
    plain(a.y, q.y);
}
__device__ inline bool g1p_eq(const g1p_t &p, const g1p_t &q) {
    using namespace fk20_device_detail;
    fk::G1P a, b;
    point(a, p);
    point(b, q);
    const bool ia = fk::f_is_zero(a.z), ib = fk::f_is_zero(b.z);
    if (ia || ib) return ia && ib;
    fk::Fp l, r;  // X1 Z2 == X2 Z1 and Y1 Z2 == Y2 Z1
    fk::f_mul(l, a.x, b.z);
    fk::f_mul(r, b.x, a.z);
    if (!fk::f_eq(l, r)) return false;
    fk::f_mul(l, a.y, b.z);
    fk::f_mul(r, b.y, a.z);
    return fk::f_eq(l, r);
}
__device__ inline bool g1p_neq(const g1p_t &p, const g1p_t &q) { return !g1p_eq(p, q); }
__device__ inline bool g1p_isInf(const g1p_t &p) {
    return fp_iszero(p.z) && fp_iszero(p.x) && fp_nonzero(p.y);
}
// Y^2 Z == X^3 + 4 Z^3, or infinity (g1p_ispoint.cu:14-60); homogeneous, so
// the words may be read as Montgomery values (both sides scale by R^-3)
__device__ inline bool g1p_isPoint(const g1p_t &p) {
    using namespace fk20_device_detail;
    fk::Fp x, y, z;
    canon(x, p.x);
    canon(y, p.y);
    canon(z, p.z);
    if (fk::f_is_zero(z)) return fk::f_is_zero(x) && !fk::f_is_zero(y);
    fk::Fp l, r, t;
    fk::f_mul(l, y, y);
    fk::f_mul(l, l, z);
    fk::f_mul(r, x, x);
    fk::f_mul(r, r, x);
    fk::f_mul(t, z, z);
    fk::f_mul(t, t, z);
    fk::f_add(t, t, t);
    fk::f_add(t, t, t);
    fk::f_add(r, r, t);
    return fk::f_eq(l, r);
}
__device__ inline void g1p_neg(g1p_t &p) {
    using namespace fk20_device_detail;
    fk::G1P a;
    point(a, p);
    fk::g1_neg(a, a);
    unpoint(p, a);
}
// (X, Y, Z) <- (sX, sY, sZ): the same point for s != 0   (g1p_scale.cu)
__device__ inline void g1p_scale(g1p_t &p, const fp_t &s) {
    fp_mul(p.x, p.x, s);
    fp_mul(p.y, p.y, s);
    fp_mul(p.z, p.z, s);
}
__device__ inline void g1p_dbl(g1p_t &p) {
    using namespace fk20_device_detail;
    fk::G1P a;
    point(a, p);
    fk::g1_dbl(a, a);
    unpoint(p, a);
}
__device__ inline void g1p_add(g1p_t &p, const g1p_t &q) {
    using namespace fk20_device_detail;
    fk::G1P a, b;
    point(a, p);
    point(b, q);
    fk::g1_add(a, a, b);
    unpoint(p, a);
}
// p += q for affine q   (g1p_add.cu:62)
__device__ inline void g1p_add(g1p_t &p, const g1a_t &q) {
    using namespace fk20_device_detail;
    fk::G1P a, b;
    point(a, p);
    point(b, q);
    fk::g1_add(a, a, b);
    unpoint(p, a);
}
__device__ inline void g1p_sub(g1p_t &p, const g1p_t &q) {
    using namespace fk20_device_detail;
    fk::G1P a, b;
    point(a, p);
    point(b, q);
    fk::g1_neg(b, b);
    fk::g1_add(a, a, b);
    unpoint(p, a);
}
// (p, q) <- (p + q, p - q)   (g1p_addsub.cu:16)
__device__ inline void g1p_addsub(g1p_t &p, g1p_t &q) {
    using namespace fk20_device_detail;
    fk::G1P a, b, s, d;
    point(a, p);
    point(b, q);
    fk::g1_add(s, a, b);
    fk::g1_neg(b, b);
    fk::g1_add(d, a, b);
    unpoint(p, s);
    unpoint(q, d);
}
// p <- [x] p, any 256-bit x   (g1p_mul.cu:18)
__device__ inline void g1p_mul(g1p_t &p, const fr_t &x) {
    using namespace fk20_device_detail;
    fk::G1P a, r;
    point(a, p);
    fk::g1_set_inf(r);
    for (int i = 255; i >= 0; i--) {
        fk::g1_dbl(r, r);
        if ((x[i >> 6] >> (i & 63)) & 1) fk::g1_add(r, r, a);
    }
    unpoint(p, r);
}
__device__ __host__ inline void g1p_print(const char *s, const g1p_t &p) {
    printf("%s #x%016llx%016llx%016llx%016llx%016llx%016llx #y%016llx%016llx%016llx%016llx%016llx%016llx "
           "#z%016llx%016llx%016llx%016llx%016llx%016llx\n",
           s, (unsigned long long)p.x[5], (unsigned long long)p.x[4], (unsigned long long)p.x[3],
           (unsigned long long)p.x[2], (unsigned long long)p.x[1], (unsigned long long)p.x[0],
           (unsigned long long)p.y[5], (unsigned long long)p.y[4], (unsigned long long)p.y[3],
           (unsigned long long)p.y[2], (unsigned long long)p.y[1], (unsigned long long)p.y[0],
           (unsigned long long)p.z[5], (unsigned long long)p.z[4], (unsigned long long)p.z[3],
           (unsigned long long)p.z[2], (unsigned long long)p.z[1], (unsigned long long)p.z[0]);
}
__device__ __host__ inline void g1a_print(const char *s, const g1a_t &a) {
    printf("%s #x%016llx%016llx%016llx%016llx%016llx%016llx #y%016llx%016llx%016llx%016llx%016llx%016llx\n", s,
           (unsigned long long)a.x[5], (unsigned long long)a.x[4], (unsigned long long)a.x[3],
           (unsigned long long)a.x[2], (unsigned long long)a.x[1], (unsigned long long)a.x[0],
           (unsigned long long)a.y[5], (unsigned long long)a.y[4], (unsigned long long)a.y[3],
           (unsigned long long)a.y[2], (unsigned long long)a.y[1], (unsigned long long)a.y[0]);
}

#endif  // FK20_DEVICE_CUH
