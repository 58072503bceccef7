// kernels_pairing.cu -- BLS12-381 pairing checks, for verifying KZG proofs.
//
// The reference verifies multiproofs with py_ecc's pairing (check_proof_multi,
// FK20Py/kzg_proofs.py:207-232; no CUDA counterpart).  This is the optimal
// ate pairing of BLS12 curves computed with the standard techniques:
//   * Fp2 = Fp[u]/(u^2 + 1), Fp6 = Fp2[v]/(v^3 - xi), Fp12 = Fp6[w]/(w^2 - v),
//     xi = 1 + u (so w^6 = xi); Karatsuba products at every level (an Fp12
//     product is 18 Fp2 products, a square 12, a product by a line 13; a
//     square in the cyclotomic subgroup, where the final exponentiation
//     works, 9 Fp2 squares).
//   * G2 on the M-type twist E': y^2 = x^3 + 4 xi, mapped into E(Fp12) by
//     psi(x', y') = (x'/w^2, y'/w^3).
//   * Miller loop over the bits of |z| = 0xd201000000010000 with T in
//     homogeneous projective coordinates (no inversions); the line through T
//     (tangent, or chord through Q) evaluated at P is c0 + c2 w^2 + c3 w^3
//     up to a factor in Fp2, which the final exponentiation removes:
//       tangent: c0 = Y^2 - 3b'Z^2, c2 = -3X^2 xP, c3 = 2YZ yP;
//       chord:   c0 = th xQ - la yQ, c2 = -th xP, c3 = la yP,
//                th = Y - yQ Z, la = X - xQ Z.
//     Both pairings of a check share one loop (one squaring of f per bit).
//     As z < 0 and the loop runs over |z|, the value is the inverse of the
//     usual normalisation: non-degenerate and bilinear all the same.
//   * Final exponentiation by 3 (p^12 - 1)/r: the easy part
//     m = f^((p^6 - 1)(p^2 + 1)) by conjugation, one inversion and a
//     Frobenius map; the hard part by the decomposition
//     3 (p^4 - p^2 + 1)/r = (z - 1)^2 (z + p)(z^2 + p^2 - 1) + 3
//     (five exponentiations by z, Frobenius maps, conjugations for the
//     inverses of the cyclotomic subgroup).  A fixed exponent coprime to r
//     keeps a check's answer the same: f^(3(p^12-1)/r) == 1 exactly when
//     f^((p^12-1)/r) == 1.
// One thread per pairing or check; field elements live in local memory and
// the Fp2 / Fp6 / Fp12 products are out-of-line routines, which keeps the
// code small.
#define FK_FP_MUL_OUTLINE 1
#include "launch.h"
#include "layout.cuh"
#include "tower.cuh"

namespace fk {

constexpr unsigned long long Z_ABS = 0xd201000000010000ull;

// ---------------------------------------------------------------- Miller loop
struct G2H {  // homogeneous projective point of the twist
    Fp2 x, y, z;
};
// T = 2T; l = (c0, c2, c3) of the tangent at T evaluated at P
static __device__ __noinline__ void dbl_step(G2H *T, Fp2 *l, const Fp *xp, const Fp *yp) {
    Fp2 B = f2s(T->y), C = f2s(T->z), E, F, XX = f2s(T->x), H, t, u, c2, c3;
    f2_xi(t, C);
    f2_mul12(E, t);  // 3 b' Z^2 = 12 xi Z^2
    f2_add(F, E, E);
    f2_add(F, F, E);  // 3 E
    H = f2m(T->y, T->z);
    f2_add(H, H, H);  // 2 Y Z
    f2_sub(t, B, E);
    f2_add(u, XX, XX);
    f2_add(u, u, XX);
    f2_mul_fp(c2, u, *xp);
    f2_neg(c2, c2);
    f2_mul_fp(c3, H, *yp);
    l[0] = t;
    l[1] = c2;
    l[2] = c3;
    t = f2m(T->x, T->y);
    f2_add(t, t, t);
    f2_sub(u, B, F);
    T->x = f2m(t, u);  // 2 X Y (B - F)
    f2_add(t, B, F);
    T->y = f2s(t);
    u = f2s(E);
    f2_mul12(u, u);
    f2_sub(T->y, T->y, u);  // (B + F)^2 - 12 E^2
    t = f2m(B, H);
    f2_add(t, t, t);
    f2_add(T->z, t, t);  // 4 B H
}
// T = T + Q (Q affine); l = (c0, c2, c3) of the chord through T and Q evaluated at P
static __device__ __noinline__ void add_step(G2H *T, Fp2 *l, const Fp2 *xq, const Fp2 *yq, const Fp *xp,
                                             const Fp *yp) {
    Fp2 th, la, t, u, c0, c2, c3, C, D, E, F, G, H;
    t = f2m(*yq, T->z);
    f2_sub(th, T->y, t);
    t = f2m(*xq, T->z);
    f2_sub(la, T->x, t);
    t = f2m(th, *xq);
    u = f2m(la, *yq);
    f2_sub(c0, t, u);
    f2_mul_fp(c2, th, *xp);
    f2_neg(c2, c2);
    f2_mul_fp(c3, la, *yp);
    l[0] = c0;
    l[1] = c2;
    l[2] = c3;
    C = f2s(th);
    D = f2s(la);
    E = f2m(la, D);
    F = f2m(T->z, C);
    G = f2m(T->x, D);
    f2_add(H, E, F);
    f2_sub(H, H, G);
    f2_sub(H, H, G);
    T->x = f2m(la, H);
    f2_sub(t, G, H);
    t = f2m(th, t);
    u = f2m(T->y, E);
    f2_sub(T->y, t, u);
    T->z = f2m(T->z, E);
}
// f = prod over the n (<= 2) pairs of their Miller values (P affine over Fp,
// Q affine on the twist, neither infinity)
static __device__ __noinline__ void miller(Fp12 *f, int n, const Fp *xp, const Fp *yp, const Fp2 *xq, const Fp2 *yq) {
    G2H T[2];
    Fp2 l[3];
#pragma unroll 1
    for (int j = 0; j < n; j++) {
        T[j].x = xq[j];
        T[j].y = yq[j];
        f2_one(T[j].z);
    }
    f12_one(*f);
#pragma unroll 1
    for (int i = 62; i >= 0; i--) {
        f12_sqr(f, f);
#pragma unroll 1
        for (int j = 0; j < n; j++) {
            dbl_step(&T[j], l, &xp[j], &yp[j]);
            f12_mul_line(f, l);
        }
        if ((Z_ABS >> i) & 1ull) {
#pragma unroll 1
            for (int j = 0; j < n; j++) {
                add_step(&T[j], l, &xq[j], &yq[j], &xp[j], &yp[j]);
                f12_mul_line(f, l);
            }
        }
    }
}

// ---------------------------------------------------------------- final exponentiation
// r = a^z (z = -|z| < 0, a in the cyclotomic subgroup, where the inverse is
// the conjugate); r may alias a
static __device__ __noinline__ void exp_z(Fp12 *r, const Fp12 *a) {
    Fp12 acc = *a;
#pragma unroll 1
    for (int i = 62; i >= 0; i--) {
        f12_cyc_sqr(&acc, &acc);
        if ((Z_ABS >> i) & 1ull) f12_mul(&acc, &acc, a);
    }
    f12_conj(*r, acc);
}
// r = f^(3 (p^12 - 1) / r)
static __device__ __noinline__ void final_exp(Fp12 *r, const Fp12 *f) {
    Fp12 m, t, a, b, c;
    f12_inv(&t, f);  // easy part: m = f^((p^6 - 1)(p^2 + 1))
    f12_conj(m, *f);
    f12_mul(&m, &m, &t);
    f12_frob(&t, &m, false);
    f12_mul(&m, &t, &m);
    exp_z(&a, &m);  // a = m^(z - 1)
    f12_conj(t, m);
    f12_mul(&a, &a, &t);
    exp_z(&t, &a);  // a = a^(z - 1)
    f12_conj(a, a);
    f12_mul(&a, &t, &a);
    exp_z(&b, &a);  // b = a^(z + p)
    f12_frob(&t, &a, true);
    f12_mul(&b, &b, &t);
    exp_z(&c, &b);  // c = b^(z^2 + p^2 - 1)
    exp_z(&c, &c);
    f12_frob(&t, &b, false);
    f12_mul(&c, &c, &t);
    f12_conj(t, b);
    f12_mul(&c, &c, &t);
    f12_cyc_sqr(&t, &m);  // times m^3
    f12_mul(&t, &t, &m);
    f12_mul(r, &c, &t);
}

// ---------------------------------------------------------------- conversions
FK_D void fp_from_words(Fp &m, const uint64_t *w) {
    Fp t;
#pragma unroll
    for (int k = 0; k < 6; k++) { t.w[2 * k] = (uint32_t)w[k]; t.w[2 * k + 1] = (uint32_t)(w[k] >> 32); }
    f_to_mont(m, t);
}
FK_D void fp_to_words(uint64_t *w, const Fp &m) {
    Fp t;
    f_from_mont(t, m);
#pragma unroll
    for (int k = 0; k < 6; k++) w[k] = (uint64_t)t.w[2 * k] | ((uint64_t)t.w[2 * k + 1] << 32);
}
// reference g1p_t -> affine (Montgomery); false for infinity
FK_D bool g1_affine(Fp &x, Fp &y, const uint64_t *g) {
    G1P p;
    g1p_from_ref(p, g);
    if (f_is_zero(p.z)) return false;
    g1_normalize(p);
    x = p.x;
    y = p.y;
    return true;
}
// g2p_t {x0, x1, y0, y1, z0, z1} (36 words, standard form) -> affine; false for infinity
FK_D bool g2_affine(Fp2 &x, Fp2 &y, const uint64_t *g) {
    Fp2 z;
    fp_from_words(x.c0, g);
    fp_from_words(x.c1, g + 6);
    fp_from_words(y.c0, g + 12);
    fp_from_words(y.c1, g + 18);
    fp_from_words(z.c0, g + 24);
    fp_from_words(z.c1, g + 30);
    if (f2_is_zero(z)) return false;
    f2_inv(&z, &z);
    x = f2m(x, z);
    y = f2m(y, z);
    return true;
}
FK_D void g2_store(uint64_t *g, const Fp2 &x, const Fp2 &y, bool inf) {
    if (inf) {
#pragma unroll 1
        for (int k = 0; k < 36; k++) g[k] = 0;
        g[12] = 1;  // (0, 1, 0)
        return;
    }
    fp_to_words(g, x.c0);
    fp_to_words(g + 6, x.c1);
    fp_to_words(g + 12, y.c0);
    fp_to_words(g + 18, y.c1);
    Fp one;
    f_set_one(one);
    fp_to_words(g + 24, one);
#pragma unroll 1
    for (int k = 30; k < 36; k++) g[k] = 0;
}

// affine G2 addition with its special cases; inf flags
static __device__ __noinline__ void g2_add(Fp2 *xr, Fp2 *yr, bool *ir, Fp2 x1, Fp2 y1, bool i1, Fp2 x2, Fp2 y2,
                                           bool i2) {
    if (i1 || i2) {
        *ir = i1 && i2;
        *xr = i1 ? x2 : x1;
        *yr = i1 ? y2 : y1;
        return;
    }
    Fp2 lam, t, u;
    if (f2_eq(x1, x2)) {
        f2_add(t, y1, y2);
        if (f2_is_zero(t)) {  // P + (-P)
            *ir = true;
            return;
        }
        t = f2m(x1, x1);
        f2_add(u, t, t);
        f2_add(t, u, t);
        f2_add(u, y1, y1);
    } else {
        f2_sub(t, y2, y1);
        f2_sub(u, x2, x1);
    }
    f2_inv(&u, &u);
    lam = f2m(t, u);
    t = f2m(lam, lam);
    f2_sub(t, t, x1);
    f2_sub(t, t, x2);
    f2_sub(u, x1, t);
    u = f2m(lam, u);
    f2_sub(*yr, u, y1);
    *xr = t;
    *ir = false;
}

// ---------------------------------------------------------------- kernels
// op 0: out[i] = e(a[i], b[i]) (12 fp_t: the 6 Fp2 coefficients of w);
// op 1: ok[i] = e(a[i], b[i]) == e(c[i], d[i]).
// bcast bit 0: b is one point for every i; bit 1: d likewise.
__global__ void __launch_bounds__(64) k_pairing(int op, uint64_t *out, uint8_t *ok, const uint64_t *a,
                                                const uint64_t *b, const uint64_t *c, const uint64_t *d,
                                                size_t count, int bcast) {
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= count) return;
    const size_t ib = (bcast & 1) ? 0 : i, id = (bcast & 2) ? 0 : i;
    Fp xp[2], yp[2];
    Fp2 xq[2], yq[2];
    int n = 0;
    if (g1_affine(xp[n], yp[n], a + 18 * i) && g2_affine(xq[n], yq[n], b + 36 * ib)) n++;
    if (op == 1 && g1_affine(xp[n], yp[n], c + 18 * i) && g2_affine(xq[n], yq[n], d + 36 * id)) {
        f_neg(yp[n], yp[n]);  // e(c, d)^-1 = e(-c, d)
        n++;
    }
    Fp12 f, e;
    if (n) miller(&f, n, xp, yp, xq, yq);
    else f12_one(f);
    final_exp(&e, &f);
    if (op == 1) {
        ok[i] = f12_is_one(e) ? 1 : 0;
        return;
    }
#pragma unroll 1
    for (int k = 0; k < 6; k++) {
        const Fp2 &v = (k & 1) ? e.a1.c[k >> 1] : e.a0.c[k >> 1];
        fp_to_words(out + 72 * i + 12 * k, v.c0);
        fp_to_words(out + 72 * i + 12 * k + 6, v.c1);
    }
}

// Interpolation for check_proof_multi (FK20Py/kzg_proofs.py:214-217): from the
// evaluations ys[k] = f(x w^k), k < l (w = w_l), the coefficients of the
// interpolation polynomial I(X) = sum_j c_j X^j, c_j = (1/l) sum_k ys[k] w^-jk
// / x^j, written as poly[32 i + j] (zero above l), and xl[i] = x^l.  Fr in
// Montgomery form inside; fr_t standard form (any representative) in,
// canonical out.
__global__ void __launch_bounds__(64) k_interp(uint64_t *poly, uint64_t *xl, const uint64_t *x, const uint64_t *ys,
                                               int log_l, size_t count) {
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int l = 1 << log_l, step = 32 >> log_l;
    Fr y[32], xm, xinv, t, acc, w, s;
#pragma unroll 1
    for (int k = 0; k < l; k++) {
        fr_from_ref(t, ys + 4 * ((size_t)l * i + k));
        f_to_mont(y[k], t);
    }
    fr_from_ref(t, x + 4 * i);
    f_to_mont(xm, t);
    f_inv(xinv, xm);
#pragma unroll
    for (int q = 0; q < 8; q++) s.w[q] = c_inv_pow2[log_l][q];  // s = (1/l) x^-j, from j = 0
#pragma unroll 1
    for (int j = 0; j < 32; j++) {
        uint64_t *dst = poly + 4 * (32 * i + j);
        if (j >= l) {
            dst[0] = dst[1] = dst[2] = dst[3] = 0;
            continue;
        }
        f_set_zero(acc);
#pragma unroll 1
        for (int k = 0; k < l; k++) {
            const int e = (j * k * step) & 31;
#pragma unroll
            for (int q = 0; q < 8; q++) w.w[q] = c_w32_inv[e][q];
            f_mul(t, y[k], w);
            f_add(acc, acc, t);
        }
        f_mul(acc, acc, s);
        f_from_mont(t, acc);
        fr_to_ref(dst, t);
        f_mul(s, s, xinv);
    }
    t = xm;
#pragma unroll 1
    for (int q = 0; q < log_l; q++) f_mul(t, t, t);
    f_from_mont(acc, t);
    fr_to_ref(xl + 4 * i, acc);
}

// G2 element-wise: 0 add, 1 dbl, 2 neg, 3 sub, 4 mul by fr_t scalar, 5 normalize,
// 6 on-curve flag (b: uint8 out)
__global__ void __launch_bounds__(64) k_g2_op(int op, uint64_t *out, const uint64_t *a, const void *b,
                                              size_t count) {
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= count) return;
    Fp2 x1, y1, x2, y2, xr, yr;
    const bool i1 = !g2_affine(x1, y1, a + 36 * i);
    bool ir = true;
    f2_zero(xr);
    f2_zero(yr);
    if (op == 6) {  // y^2 == x^3 + 4 xi, or infinity
        bool on = true;
        if (!i1) {
            Fp2 l = f2m(y1, y1), r = f2m(f2m(x1, x1), x1), bb;
            f_set_zero(bb.c0);
            f_set_zero(bb.c1);
            bb.c0.w[0] = 4;
            Fp t;
            f_to_mont(t, bb.c0);
            bb.c0 = t;
            bb.c1 = t;
            f2_add(r, r, bb);
            on = f2_eq(l, r);
        }
        ((uint8_t *)b)[i] = on ? 1 : 0;
        return;
    }
    if (op == 0 || op == 3) {
        const bool i2 = !g2_affine(x2, y2, (const uint64_t *)b + 36 * i);
        if (op == 3) f2_neg(y2, y2);
        g2_add(&xr, &yr, &ir, x1, y1, i1, x2, y2, i2);
    } else if (op == 1) {
        g2_add(&xr, &yr, &ir, x1, y1, i1, x1, y1, i1);
    } else if (op == 2) {
        xr = x1;
        f2_neg(yr, y1);
        ir = i1;
    } else if (op == 4) {
        const uint64_t *s = (const uint64_t *)b + 4 * i;
#pragma unroll 1
        for (int k = 255; k >= 0; k--) {
            g2_add(&xr, &yr, &ir, xr, yr, ir, xr, yr, ir);
            if ((s[k >> 6] >> (k & 63)) & 1ull) g2_add(&xr, &yr, &ir, xr, yr, ir, x1, y1, i1);
        }
    } else {
        xr = x1;
        yr = y1;
        ir = i1;
    }
    g2_store(out + 36 * i, xr, yr, ir);
}

void launch_pairing(int op, uint64_t *out, uint8_t *ok, const uint64_t *a, const uint64_t *b, const uint64_t *c,
                    const uint64_t *d, size_t count, cudaStream_t st, int bcast) {
    k_pairing<<<blocks_for(count, 64), 64, 0, st>>>(op, out, ok, a, b, c, d, count, bcast);
}
void launch_interp(uint64_t *poly, uint64_t *xl, const uint64_t *x, const uint64_t *ys, int log_l, size_t count,
                   cudaStream_t st) {
    k_interp<<<blocks_for(count, 64), 64, 0, st>>>(poly, xl, x, ys, log_l, count);
}
void launch_g2_op(int op, uint64_t *out, const uint64_t *a, const void *b, size_t count, cudaStream_t st) {
    k_g2_op<<<blocks_for(count, 64), 64, 0, st>>>(op, out, a, b, count);
}

}  // namespace fk
