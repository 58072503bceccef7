// tower.cuh -- the extension-field tower of the BLS12-381 pairing:
// Fp2 = Fp[u]/(u^2 + 1), Fp6 = Fp2[v]/(v^3 - xi), Fp12 = Fp6[w]/(w^2 - v),
// xi = 1 + u (so w^6 = xi), with Karatsuba products at every level, the
// Frobenius maps, the cyclotomic squaring of the final exponentiation and the
// sparse product by a Miller-loop line.  Used by kernels_pairing.cu (and by a
// test probe that compiles the same routines).  The translation unit defines
// FK_FP_MUL_OUTLINE before including layout.cuh / g1.cuh, so every Fp product
// is one shared out-of-line routine.
#pragma once
#include "g1.cuh"

namespace fk {

#include "pairing_consts.inc"

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
// 3 Fp products.  The out-of-line Fp2 routines take and return values, not
// pointers: with pointer arguments (r may alias a or b) some code
// arrangements of their callers -- an Fp6 sum as a rolled loop before an
// in-place product by a line -- gave wrong values in the GPU build while the
// source is right (it is right on the host and unoptimised); with values they
// give the right ones in every arrangement tried (tests/host/tower_probe.cu).
static __device__ __noinline__ Fp2 f2_mul_v(Fp2 a, Fp2 b) {
    Fp t0, t1, s0, s1;
    Fp2 r;
    fp_mul(t0, a.c0, b.c0);
    fp_mul(t1, a.c1, b.c1);
    f_add(s0, a.c0, a.c1);
    f_add(s1, b.c0, b.c1);
    fp_mul(s0, s0, s1);
    f_sub(s0, s0, t0);
    f_sub(r.c1, s0, t1);
    f_sub(r.c0, t0, t1);
    return r;
}
// (a0 + a1 u)^2 = (a0 + a1)(a0 - a1) + 2 a0 a1 u
static __device__ __noinline__ Fp2 f2_sqr_v(Fp2 a) {
    Fp s, d, t;
    Fp2 r;
    f_add(s, a.c0, a.c1);
    f_sub(d, a.c0, a.c1);
    fp_mul(t, a.c0, a.c1);
    fp_mul(r.c0, s, d);
    f_add(r.c1, t, t);
    return r;
}
// r may alias a or b
FK_D void f2_mul(Fp2 *r, const Fp2 *a, const Fp2 *b) { *r = f2_mul_v(*a, *b); }
FK_D void f2_sqr(Fp2 *r, const Fp2 *a) { *r = f2_sqr_v(*a); }
FK_D Fp2 f2m(const Fp2 &a, const Fp2 &b) { return f2_mul_v(a, b); }
FK_D Fp2 f2s(const Fp2 &a) { return f2_sqr_v(a); }
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

}  // namespace fk
