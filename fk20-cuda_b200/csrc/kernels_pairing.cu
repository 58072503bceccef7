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

namespace fk {

#include "pairing_consts.inc"

constexpr unsigned long long Z_ABS = 0xd201000000010000ull;

struct Fp2 {
    Fp c0, c1;
};
struct Fp6 {  // c[0] + c[1] v + c[2] v^2
    Fp2 c[3];
};
struct Fp12 {  // a0 + a1 w; the coefficient of w^k is a0.c[k/2] (k even) or a1.c[k/2] (k odd)
    Fp6 a0, a1;
};

// ---------------------------------------------------------------- Fp2
FK_D void f2_add(Fp2 &r, const Fp2 &a, const Fp2 &b) { f_add(r.c0, a.c0, b.c0); f_add(r.c1, a.c1, b.c1); }
FK_D void f2_sub(Fp2 &r, const Fp2 &a, const Fp2 &b) { f_sub(r.c0, a.c0, b.c0); f_sub(r.c1, a.c1, b.c1); }
FK_D void f2_neg(Fp2 &r, const Fp2 &a) { f_neg(r.c0, a.c0); f_neg(r.c1, a.c1); }
FK_D void f2_conj(Fp2 &r, const Fp2 &a) { r.c0 = a.c0; f_neg(r.c1, a.c1); }
FK_D bool f2_is_zero(const Fp2 &a) { return f_is_zero(a.c0) && f_is_zero(a.c1); }
FK_D bool f2_eq(const Fp2 &a, const Fp2 &b) { return f_eq(a.c0, b.c0) && f_eq(a.c1, b.c1); }
FK_D void f2_zero(Fp2 &r) { f_set_zero(r.c0); f_set_zero(r.c1); }
FK_D void f2_one(Fp2 &r) { f_set_one(r.c0); f_set_zero(r.c1); }
// a (1 + u)
FK_D void f2_xi(Fp2 &r, const Fp2 &a) {
    Fp t;
    f_sub(t, a.c0, a.c1);
    f_add(r.c1, a.c0, a.c1);
    r.c0 = t;
}
// 3 Fp products; r may alias a or b
static __device__ __noinline__ void f2_mul(Fp2 *r, const Fp2 *a, const Fp2 *b) {
    Fp t0, t1, s0, s1;
    fp_mul(t0, a->c0, b->c0);
    fp_mul(t1, a->c1, b->c1);
    f_add(s0, a->c0, a->c1);
    f_add(s1, b->c0, b->c1);
    fp_mul(s0, s0, s1);
    f_sub(s0, s0, t0);
    f_sub(r->c1, s0, t1);
    f_sub(r->c0, t0, t1);
}
// (a0 + a1 u)^2 = (a0 + a1)(a0 - a1) + 2 a0 a1 u
static __device__ __noinline__ void f2_sqr(Fp2 *r, const Fp2 *a) {
    Fp s, d, t;
    f_add(s, a->c0, a->c1);
    f_sub(d, a->c0, a->c1);
    fp_mul(t, a->c0, a->c1);
    fp_mul(r->c0, s, d);
    f_add(r->c1, t, t);
}
FK_D Fp2 f2m(const Fp2 &a, const Fp2 &b) {
    Fp2 r;
    f2_mul(&r, &a, &b);
    return r;
}
FK_D Fp2 f2s(const Fp2 &a) {
    Fp2 r;
    f2_sqr(&r, &a);
    return r;
}
FK_D void f2_mul_fp(Fp2 &r, const Fp2 &a, const Fp &s) {
    fp_mul(r.c0, a.c0, s);
    fp_mul(r.c1, a.c1, s);
}
// 12 a (a multiple of 2, 4, 8 by additions)
FK_D void f2_mul12(Fp2 &r, const Fp2 &a) {
    Fp2 t4, t8;
    f2_add(t4, a, a);
    f2_add(t4, t4, t4);
    f2_add(t8, t4, t4);
    f2_add(r, t8, t4);
}
// 1 / (a0 + a1 u) = (a0 - a1 u) / (a0^2 + a1^2); inv(0) = 0
static __device__ __noinline__ void f2_inv(Fp2 *r, const Fp2 *a) {
    Fp n, t;
    fp_mul(n, a->c0, a->c0);
    fp_mul(t, a->c1, a->c1);
    f_add(n, n, t);
    f_inv(n, n);
    fp_mul(r->c0, a->c0, n);
    fp_mul(t, a->c1, n);
    f_neg(r->c1, t);
}

// ---------------------------------------------------------------- Fp6
FK_D void f6_add(Fp6 &r, const Fp6 &a, const Fp6 &b) {
#pragma unroll 1
    for (int k = 0; k < 3; k++) f2_add(r.c[k], a.c[k], b.c[k]);
}
FK_D void f6_sub(Fp6 &r, const Fp6 &a, const Fp6 &b) {
#pragma unroll 1
    for (int k = 0; k < 3; k++) f2_sub(r.c[k], a.c[k], b.c[k]);
}
FK_D void f6_neg(Fp6 &r, const Fp6 &a) {
#pragma unroll 1
    for (int k = 0; k < 3; k++) f2_neg(r.c[k], a.c[k]);
}
FK_D void f6_zero(Fp6 &r) {
#pragma unroll 1
    for (int k = 0; k < 3; k++) f2_zero(r.c[k]);
}
FK_D bool f6_is_zero(const Fp6 &a) { return f2_is_zero(a.c[0]) && f2_is_zero(a.c[1]) && f2_is_zero(a.c[2]); }
// a v (v^3 = xi); r may alias a
FK_D void f6_mulv(Fp6 &r, const Fp6 &a) {
    Fp2 t;
    f2_xi(t, a.c[2]);
    r.c[2] = a.c[1];
    r.c[1] = a.c[0];
    r.c[0] = t;
}
// Karatsuba, 6 Fp2 products; r may alias x or y
static __device__ __noinline__ void f6_mul(Fp6 *r, const Fp6 *x, const Fp6 *y) {
    Fp2 t0, t1, t2, s, u, c0, c1;
    f2_mul(&t0, &x->c[0], &y->c[0]);
    f2_mul(&t1, &x->c[1], &y->c[1]);
    f2_mul(&t2, &x->c[2], &y->c[2]);
    f2_add(s, x->c[1], x->c[2]);  // c0 = t0 + xi ((x1 + x2)(y1 + y2) - t1 - t2)
    f2_add(u, y->c[1], y->c[2]);
    f2_mul(&s, &s, &u);
    f2_sub(s, s, t1);
    f2_sub(s, s, t2);
    f2_xi(s, s);
    f2_add(c0, t0, s);
    f2_add(s, x->c[0], x->c[1]);  // c1 = (x0 + x1)(y0 + y1) - t0 - t1 + xi t2
    f2_add(u, y->c[0], y->c[1]);
    f2_mul(&s, &s, &u);
    f2_sub(s, s, t0);
    f2_sub(s, s, t1);
    f2_xi(u, t2);
    f2_add(c1, s, u);
    f2_add(s, x->c[0], x->c[2]);  // c2 = (x0 + x2)(y0 + y2) - t0 - t2 + t1
    f2_add(u, y->c[0], y->c[2]);
    f2_mul(&s, &s, &u);
    f2_sub(s, s, t0);
    f2_sub(s, s, t2);
    f2_add(r->c[2], s, t1);
    r->c[0] = c0;
    r->c[1] = c1;
}
// (t0 + t1 v + t2 v^2) / N with t0 = x0^2 - xi x1 x2, t1 = xi x2^2 - x0 x1,
// t2 = x1^2 - x0 x2, N = x0 t0 + xi (x2 t1 + x1 t2); inv(0) = 0
static __device__ __noinline__ void f6_inv(Fp6 *r, const Fp6 *x) {
    Fp2 t0, t1, t2, s, n;
    t0 = f2s(x->c[0]);
    s = f2m(x->c[1], x->c[2]);
    f2_xi(s, s);
    f2_sub(t0, t0, s);
    t1 = f2s(x->c[2]);
    f2_xi(t1, t1);
    s = f2m(x->c[0], x->c[1]);
    f2_sub(t1, t1, s);
    t2 = f2s(x->c[1]);
    s = f2m(x->c[0], x->c[2]);
    f2_sub(t2, t2, s);
    n = f2m(x->c[2], t1);
    s = f2m(x->c[1], t2);
    f2_add(n, n, s);
    f2_xi(n, n);
    s = f2m(x->c[0], t0);
    f2_add(n, n, s);
    f2_inv(&n, &n);
    r->c[0] = f2m(t0, n);
    r->c[1] = f2m(t1, n);
    r->c[2] = f2m(t2, n);
}

// ---------------------------------------------------------------- Fp12
FK_D void f12_one(Fp12 &r) {
    f6_zero(r.a0);
    f6_zero(r.a1);
    f2_one(r.a0.c[0]);
}
FK_D bool f12_is_one(const Fp12 &a) {
    Fp2 one;
    f2_one(one);
    return f2_eq(a.a0.c[0], one) && f2_is_zero(a.a0.c[1]) && f2_is_zero(a.a0.c[2]) && f6_is_zero(a.a1);
}
// f^(p^6): the conjugate over Fp6 (the inverse in the cyclotomic subgroup)
FK_D void f12_conj(Fp12 &r, const Fp12 &a) {
    r.a0 = a.a0;
    f6_neg(r.a1, a.a1);
}
// 3 Fp6 products; r may alias a or b
static __device__ __noinline__ void f12_mul(Fp12 *r, const Fp12 *a, const Fp12 *b) {
    Fp6 t0, t1, s, u;
    f6_mul(&t0, &a->a0, &b->a0);
    f6_mul(&t1, &a->a1, &b->a1);
    f6_add(s, a->a0, a->a1);
    f6_add(u, b->a0, b->a1);
    f6_mul(&s, &s, &u);
    f6_sub(s, s, t0);
    f6_sub(r->a1, s, t1);
    f6_mulv(t1, t1);
    f6_add(r->a0, t0, t1);
}
// (a0 + a1 w)^2 = ((a0 + a1)(a0 + v a1) - t - v t) + 2 t w, t = a0 a1: 2 Fp6 products
static __device__ __noinline__ void f12_sqr(Fp12 *r, const Fp12 *a) {
    Fp6 t, s, u;
    f6_mul(&t, &a->a0, &a->a1);
    f6_add(s, a->a0, a->a1);
    f6_mulv(u, a->a1);
    f6_add(u, a->a0, u);
    f6_mul(&s, &s, &u);
    f6_sub(s, s, t);
    f6_mulv(u, t);
    f6_sub(r->a0, s, u);
    f6_add(r->a1, t, t);
}
// (a0 + a1 w)^-1 = (a0 - a1 w) / (a0^2 - v a1^2)
static __device__ __noinline__ void f12_inv(Fp12 *r, const Fp12 *a) {
    Fp6 s, t;
    f6_mul(&s, &a->a0, &a->a0);
    f6_mul(&t, &a->a1, &a->a1);
    f6_mulv(t, t);
    f6_sub(s, s, t);
    f6_inv(&s, &s);
    f6_mul(&r->a0, &a->a0, &s);
    f6_neg(t, a->a1);
    f6_mul(&r->a1, &t, &s);
}
FK_D void frob_coef(Fp2 &g, const uint32_t (*c)[12]) {
#pragma unroll
    for (int i = 0; i < 12; i++) {
        g.c0.w[i] = c[0][i];
        g.c1.w[i] = c[1][i];
    }
}
// a^p (conj = true, coefficients c_frob1) or a^(p^2) (conj = false, c_frob2):
// sum_k a_k^(p^j) g_k w^k
static __device__ __noinline__ void f12_frob(Fp12 *r, const Fp12 *a, bool conj) {
    const uint32_t(*tab)[2][12] = conj ? c_frob1 : c_frob2;
#pragma unroll 1
    for (int k = 0; k < 6; k++) {
        const Fp2 &src = (k & 1) ? a->a1.c[k >> 1] : a->a0.c[k >> 1];
        Fp2 &dst = (k & 1) ? r->a1.c[k >> 1] : r->a0.c[k >> 1];
        Fp2 x, g;
        if (conj) f2_conj(x, src);
        else x = src;
        frob_coef(g, tab[k]);
        f2_mul(&dst, &x, &g);
    }
}

// x^2 in Fp4 = Fp2[s]/(s^2 - xi) for x = (x0, x1) = x0 + x1 s: (x0^2 + xi x1^2, 2 x0 x1)
FK_D void f4_sqr(Fp2 &r0, Fp2 &r1, const Fp2 &x0, const Fp2 &x1) {
    Fp2 a = f2s(x0), b = f2s(x1), t;
    f2_add(t, x0, x1);
    t = f2s(t);
    f2_sub(t, t, a);
    f2_sub(r1, t, b);
    f2_xi(b, b);
    f2_add(r0, a, b);
}
// 3 a - 2 b = a + 2 (a - b) and 3 a + 2 b = a + 2 (a + b)
FK_D void f2_3a_2b(Fp2 &r, const Fp2 &a, const Fp2 &b, bool minus) {
    Fp2 t;
    if (minus) f2_sub(t, a, b);
    else f2_add(t, a, b);
    f2_add(t, t, t);
    f2_add(r, a, t);
}
// r = a^2 for a in the cyclotomic subgroup (a^(p^6 + 1) = 1, a^(p^4 - p^2 + 1)
// = 1), as Granger and Scott square there: with Fp12 = Fp4[w]/(w^3 - s),
// s = w^3, a = g0 + g1 w + g2 w^2 (g0 = (w0, w3), g1 = (w1, w4), g2 = (w2, w5)):
// a^2 = (3 g0^2 - 2 conj g0) + (3 s g2^2 + 2 conj g1) w + (3 g1^2 - 2 conj g2) w^2,
// conj the Fp4 conjugate (x0, x1) -> (x0, -x1): 9 Fp2 squares instead of 12
// Fp2 products; r may alias a
static __device__ __noinline__ void f12_cyc_sqr(Fp12 *r, const Fp12 *a) {
    Fp2 A0, A1, B0, B1, C0, C1, o[6];
    f4_sqr(A0, A1, a->a0.c[0], a->a1.c[1]);
    f4_sqr(B0, B1, a->a1.c[0], a->a0.c[2]);
    f4_sqr(C0, C1, a->a0.c[1], a->a1.c[2]);
    f2_3a_2b(o[0], A0, a->a0.c[0], true);   // w^0
    f2_3a_2b(o[3], A1, a->a1.c[1], false);  // w^3
    f2_xi(C1, C1);
    f2_3a_2b(o[1], C1, a->a1.c[0], false);  // w^1: 3 xi C1 + 2 g1.0
    f2_3a_2b(o[4], C0, a->a0.c[2], true);   // w^4: 3 C0 - 2 g1.1
    f2_3a_2b(o[2], B0, a->a0.c[1], true);   // w^2
    f2_3a_2b(o[5], B1, a->a1.c[2], false);  // w^5
    r->a0.c[0] = o[0];
    r->a1.c[0] = o[1];
    r->a0.c[1] = o[2];
    r->a1.c[1] = o[3];
    r->a0.c[2] = o[4];
    r->a1.c[2] = o[5];
}

// r = x (c0 + c1 v): 5 Fp2 products; r may alias x
FK_D void f6_mul01(Fp6 &r, const Fp6 &x, const Fp2 &c0, const Fp2 &c1) {
    Fp2 t0 = f2m(x.c[0], c0), t1 = f2m(x.c[1], c1), u, v, r0, r1;
    u = f2m(x.c[2], c1);
    f2_xi(u, u);
    f2_add(r0, t0, u);
    f2_add(u, x.c[0], x.c[1]);
    f2_add(v, c0, c1);
    u = f2m(u, v);
    f2_sub(u, u, t0);
    f2_sub(r1, u, t1);
    u = f2m(x.c[2], c0);
    f2_add(r.c[2], t1, u);
    r.c[0] = r0;
    r.c[1] = r1;
}
// r = x (c1 v): 3 Fp2 products; r may alias x
FK_D void f6_mul1(Fp6 &r, const Fp6 &x, const Fp2 &c1) {
    Fp2 t = f2m(x.c[2], c1);
    f2_xi(t, t);
    r.c[2] = f2m(x.c[1], c1);
    r.c[1] = f2m(x.c[0], c1);
    r.c[0] = t;
}
// Fp6 sums written out, not as a loop: with the rolled loops of f6_add /
// f6_sub after the products below, the GPU build of f12_mul_line gave wrong
// odd coefficients (the same source is right on the host, and right with
// the sums unrolled or placed before the products)
FK_D void f6_add3(Fp6 &r, const Fp6 &a, const Fp6 &b) {
    f2_add(r.c[0], a.c[0], b.c[0]);
    f2_add(r.c[1], a.c[1], b.c[1]);
    f2_add(r.c[2], a.c[2], b.c[2]);
}
FK_D void f6_sub3(Fp6 &r, const Fp6 &a, const Fp6 &b) {
    f2_sub(r.c[0], a.c[0], b.c[0]);
    f2_sub(r.c[1], a.c[1], b.c[1]);
    f2_sub(r.c[2], a.c[2], b.c[2]);
}
// f = f (c0 + c2 w^2 + c3 w^3), l = (c0, c2, c3): the sparse product by a
// line, 13 Fp2 products instead of 18
static __device__ __noinline__ void f12_mul_line(Fp12 *f, const Fp2 *l) {
    Fp6 t0, t1, s;
    Fp2 c23;
    f6_mul01(t0, f->a0, l[0], l[1]);
    f6_mul1(t1, f->a1, l[2]);
    f6_add3(s, f->a0, f->a1);
    f2_add(c23, l[1], l[2]);
    f6_mul01(s, s, l[0], c23);
    f6_sub3(s, s, t0);
    f6_sub3(f->a1, s, t1);
    f6_mulv(t1, t1);
    f6_add3(f->a0, t0, t1);
}

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
