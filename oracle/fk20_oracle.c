/*
 * fk20_oracle.c -- CPU restatement of the FK20 reference algorithm.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA
 * engine.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline /
 * reference arm may load it; the product library never links or calls it.
 *
 * What it restates (file:line in lCardosoSantos/FK20-CUDA):
 *   - FK20 data-availability multi-proof: FK20Py/fk20_multi_cuda.py:67-246
 *       xext_fft[i] = FFT_2k(setup[n-l-1-i :: -l] ++ [inf] ++ [inf]*k)   (:104-109, fk20_single.py:45-58)
 *       toeplitz coefficients of row i                                   (:139-146)
 *       hext_fft = sum_i tc_fft[i] (.) xext_fft[i]                        (:163-171, fk20_single.py:60-76)
 *       h = IFFT(hext_fft)[:k] ; h ++= [inf]*k ; h_fft = FFT(h)            (:195-223, fk20_single.py:78-84)
 *   - radix-2 FFT over Fr and over G1 with the same index convention and
 *     the n^-1 scaling of the inverse: FFT/fft.py:17-55
 *   - setup s_i = tau^i * G1 : FFT/kzg_proofs.py:22-30
 *   - root of unity of order m = 5^((r-1)/m) : FFT/kzg_proofs.py:39-44
 *   - G1 group law of y^2 = x^3 + 4 over Fp, generator: g1p.cu:108-129,
 *     g1p_ispoint.cu:34-60; infinity encoded (0,1,0): g1p.cu:95-100,
 *     FK20Py/toByte.py:40-46.
 *   - toeplitz gather as launched by the CUDA reference:
 *     fk20_poly2toeplitz_coefficients.cu:25-58 (identical to the Python slice).
 *   - scalar multiplication = double-and-add over the integer scalar,
 *     g1p_mul.cu:18-67 (same group element as py_ecc's multiply).
 *
 * Internal representation: 64-bit limbs, Montgomery form (R = 2^384 for Fp,
 * R = 2^256 for Fr), Jacobian coordinates for G1 with explicit exceptional
 * cases.  This deliberately differs from the engine (32-bit limbs, complete
 * homogeneous formulas), so the two implementations check each other.
 * I/O uses the reference's layout: little-endian uint64 limbs in standard
 * (non-Montgomery) form; fr_t = 4 limbs, fp_t = 6 limbs, g1p_t = {x,y,z}
 * homogeneous projective (x = X/Z, y = Y/Z), infinity = (0,1,0).
 */
#include <stdint.h>
#include <string.h>
#include <stdlib.h>
#include <pthread.h>

typedef unsigned __int128 u128;

/* ------------------------------------------------------------------------- */
/* moduli                                                                     */
/* ------------------------------------------------------------------------- */

static const uint64_t P_[6] = {
    0xb9feffffffffaaabULL, 0x1eabfffeb153ffffULL, 0x6730d2a0f6b0f624ULL,
    0x64774b84f38512bfULL, 0x4b1ba7b6434bacd7ULL, 0x1a0111ea397fe69aULL};
static const uint64_t R_[4] = {
    0xffffffff00000001ULL, 0x53bda402fffe5bfeULL, 0x3339d80809a1d805ULL,
    0x73eda753299d7d48ULL};

typedef struct { uint64_t v[6]; } fp;
typedef struct { uint64_t v[4]; } fr;

/* Montgomery constants, derived at start-up (no transcribed tables). */
static uint64_t P_INV, R_INV;      /* -m^-1 mod 2^64 */
static fp FP_ONE, FP_R2;           /* R mod p, R^2 mod p */
static fr FR_ONE, FR_R2;
static int g_init = 0;

static uint64_t neg_inv64(uint64_t m0) {
    uint64_t x = 1;                  /* Newton iteration for m0^-1 mod 2^64 */
    for (int i = 0; i < 7; i++) x *= 2 - m0 * x;
    return (uint64_t)0 - x;
}

static int geq_n(const uint64_t *a, const uint64_t *b, int n) {
    for (int i = n - 1; i >= 0; i--) {
        if (a[i] != b[i]) return a[i] > b[i];
    }
    return 1;
}
static uint64_t sub_n(uint64_t *z, const uint64_t *a, const uint64_t *b, int n) {
    uint64_t br = 0;
    for (int i = 0; i < n; i++) {
        u128 d = (u128)a[i] - b[i] - br;
        z[i] = (uint64_t)d;
        br = (uint64_t)(d >> 64) ? 1 : 0;
    }
    return br;
}
static uint64_t add_n(uint64_t *z, const uint64_t *a, const uint64_t *b, int n) {
    u128 c = 0;
    for (int i = 0; i < n; i++) {
        c += (u128)a[i] + b[i];
        z[i] = (uint64_t)c;
        c >>= 64;
    }
    return (uint64_t)c;
}

/* CIOS Montgomery product z = a*b*2^(-64n) mod m, for a*b < m*2^(64n). */
static void mont_mul_n(uint64_t *z, const uint64_t *a, const uint64_t *b,
                       const uint64_t *m, uint64_t minv, int n) {
    uint64_t t[8] = {0};
    for (int i = 0; i < n; i++) {
        u128 c = 0;
        for (int j = 0; j < n; j++) {
            c += (u128)t[j] + (u128)a[j] * b[i];
            t[j] = (uint64_t)c;
            c >>= 64;
        }
        c += t[n];
        t[n] = (uint64_t)c;
        t[n + 1] = (uint64_t)(c >> 64);
        uint64_t q = t[0] * minv;
        c = (u128)t[0] + (u128)q * m[0];
        c >>= 64;
        for (int j = 1; j < n; j++) {
            c += (u128)t[j] + (u128)q * m[j];
            t[j - 1] = (uint64_t)c;
            c >>= 64;
        }
        c += t[n];
        t[n - 1] = (uint64_t)c;
        t[n] = t[n + 1] + (uint64_t)(c >> 64);
    }
    if (t[n] || geq_n(t, m, n)) sub_n(t, t, m, n);
    memcpy(z, t, 8 * n);
}

/* ---- Fp ---------------------------------------------------------------- */
static void fp_mul(fp *z, const fp *a, const fp *b) { mont_mul_n(z->v, a->v, b->v, P_, P_INV, 6); }
static void fp_sqr(fp *z, const fp *a) { mont_mul_n(z->v, a->v, a->v, P_, P_INV, 6); }
static void fp_add(fp *z, const fp *a, const fp *b) {
    uint64_t c = add_n(z->v, a->v, b->v, 6);
    if (c || geq_n(z->v, P_, 6)) sub_n(z->v, z->v, P_, 6);
}
static void fp_sub(fp *z, const fp *a, const fp *b) {
    if (sub_n(z->v, a->v, b->v, 6)) add_n(z->v, z->v, P_, 6);
}
static void fp_neg(fp *z, const fp *a) {
    fp zero = {{0}};
    fp_sub(z, &zero, a);
}
static int fp_is0(const fp *a) {
    uint64_t o = 0;
    for (int i = 0; i < 6; i++) o |= a->v[i];
    return o == 0;
}
static int fp_equal(const fp *a, const fp *b) { return memcmp(a, b, sizeof(fp)) == 0; }
/* any 384-bit representative -> Montgomery form (a*R2 < 2^384 * p, so one product suffices) */
static void fp_from_std(fp *z, const uint64_t *x) { fp t; memcpy(t.v, x, 48); fp_mul(z, &t, &FP_R2); }
static void fp_to_std(uint64_t *z, const fp *a) { fp one = {{1}}; fp t; fp_mul(&t, a, &one); memcpy(z, t.v, 48); }
static void fp_pow(fp *z, const fp *a, const uint64_t *e, int nlimbs) {
    fp acc = FP_ONE;
    for (int i = 64 * nlimbs - 1; i >= 0; i--) {
        fp_sqr(&acc, &acc);
        if ((e[i / 64] >> (i % 64)) & 1) fp_mul(&acc, &acc, a);
    }
    *z = acc;
}
static void fp_inv(fp *z, const fp *a) {   /* Fermat: a^(p-2); inv(0) = 0 */
    uint64_t e[6];
    memcpy(e, P_, 48);
    e[0] -= 2;
    fp_pow(z, a, e, 6);
}

/* ---- Fr ---------------------------------------------------------------- */
static void fr_mul(fr *z, const fr *a, const fr *b) { mont_mul_n(z->v, a->v, b->v, R_, R_INV, 4); }
static void fr_add(fr *z, const fr *a, const fr *b) {
    uint64_t c = add_n(z->v, a->v, b->v, 4);
    if (c || geq_n(z->v, R_, 4)) sub_n(z->v, z->v, R_, 4);
}
static void fr_sub(fr *z, const fr *a, const fr *b) {
    if (sub_n(z->v, a->v, b->v, 4)) add_n(z->v, z->v, R_, 4);
}
static void fr_from_std(fr *z, const uint64_t *x) { fr t; memcpy(t.v, x, 32); fr_mul(z, &t, &FR_R2); }
static void fr_to_std(uint64_t *z, const fr *a) { fr one = {{1}}; fr t; fr_mul(&t, a, &one); memcpy(z, t.v, 32); }
static void fr_pow(fr *z, const fr *a, const uint64_t *e, int nlimbs) {
    fr acc = FR_ONE;
    for (int i = 64 * nlimbs - 1; i >= 0; i--) {
        fr_mul(&acc, &acc, &acc);
        if ((e[i / 64] >> (i % 64)) & 1) fr_mul(&acc, &acc, a);
    }
    *z = acc;
}
static void fr_inv(fr *z, const fr *a) {
    uint64_t e[4];
    memcpy(e, R_, 32);
    e[0] -= 2;
    fr_pow(z, a, e, 4);
}

static void init_consts(void) {
    if (g_init) return;
    P_INV = neg_inv64(P_[0]);
    R_INV = neg_inv64(R_[0]);
    /* R mod m by 64n doublings of 1 mod m; R^2 mod m by 64n more. */
    uint64_t t[6] = {1, 0, 0, 0, 0, 0};
    for (int i = 0; i < 384; i++) {
        uint64_t c = add_n(t, t, t, 6);
        if (c || geq_n(t, P_, 6)) sub_n(t, t, P_, 6);
    }
    memcpy(FP_ONE.v, t, 48);
    for (int i = 0; i < 384; i++) {
        uint64_t c = add_n(t, t, t, 6);
        if (c || geq_n(t, P_, 6)) sub_n(t, t, P_, 6);
    }
    memcpy(FP_R2.v, t, 48);
    uint64_t u[4] = {1, 0, 0, 0};
    for (int i = 0; i < 256; i++) {
        uint64_t c = add_n(u, u, u, 4);
        if (c || geq_n(u, R_, 4)) sub_n(u, u, R_, 4);
    }
    memcpy(FR_ONE.v, u, 32);
    for (int i = 0; i < 256; i++) {
        uint64_t c = add_n(u, u, u, 4);
        if (c || geq_n(u, R_, 4)) sub_n(u, u, R_, 4);
    }
    memcpy(FR_R2.v, u, 32);
    g_init = 1;
}

/* ------------------------------------------------------------------------- */
/* G1, Jacobian coordinates (x = X/Z^2, y = Y/Z^3), infinity: Z = 0          */
/* ------------------------------------------------------------------------- */
typedef struct { fp X, Y, Z; } jac;

static void jac_set_inf(jac *p) { memset(p, 0, sizeof *p); p->X = FP_ONE; p->Y = FP_ONE; }
static int jac_is_inf(const jac *p) { return fp_is0(&p->Z); }

static void jac_dbl(jac *r, const jac *p) {      /* dbl-2009-l, a = 0 */
    if (jac_is_inf(p) || fp_is0(&p->Y)) { jac_set_inf(r); return; }
    fp A, B, C, D, E, F, t;
    fp_sqr(&A, &p->X);
    fp_sqr(&B, &p->Y);
    fp_sqr(&C, &B);
    fp_add(&t, &p->X, &B);
    fp_sqr(&t, &t);
    fp_sub(&t, &t, &A);
    fp_sub(&t, &t, &C);
    fp_add(&D, &t, &t);
    fp_add(&E, &A, &A);
    fp_add(&E, &E, &A);
    fp_sqr(&F, &E);
    jac o;
    fp_add(&t, &D, &D);
    fp_sub(&o.X, &F, &t);
    fp_sub(&t, &D, &o.X);
    fp_mul(&t, &E, &t);
    fp C8;
    fp_add(&C8, &C, &C);
    fp_add(&C8, &C8, &C8);
    fp_add(&C8, &C8, &C8);
    fp_sub(&o.Y, &t, &C8);
    fp_mul(&o.Z, &p->Y, &p->Z);
    fp_add(&o.Z, &o.Z, &o.Z);
    *r = o;
}

static void jac_add(jac *r, const jac *p, const jac *q) {   /* add-2007-bl */
    if (jac_is_inf(p)) { *r = *q; return; }
    if (jac_is_inf(q)) { *r = *p; return; }
    fp Z1Z1, Z2Z2, U1, U2, S1, S2, H, I, J, rr, V, t;
    fp_sqr(&Z1Z1, &p->Z);
    fp_sqr(&Z2Z2, &q->Z);
    fp_mul(&U1, &p->X, &Z2Z2);
    fp_mul(&U2, &q->X, &Z1Z1);
    fp_mul(&S1, &p->Y, &q->Z);
    fp_mul(&S1, &S1, &Z2Z2);
    fp_mul(&S2, &q->Y, &p->Z);
    fp_mul(&S2, &S2, &Z1Z1);
    fp_sub(&H, &U2, &U1);
    fp_sub(&rr, &S2, &S1);
    if (fp_is0(&H)) {
        if (fp_is0(&rr)) { jac_dbl(r, p); return; }
        jac_set_inf(r);
        return;
    }
    fp_add(&rr, &rr, &rr);
    fp_add(&I, &H, &H);
    fp_sqr(&I, &I);
    fp_mul(&J, &H, &I);
    fp_mul(&V, &U1, &I);
    jac o;
    fp_sqr(&o.X, &rr);
    fp_sub(&o.X, &o.X, &J);
    fp_sub(&o.X, &o.X, &V);
    fp_sub(&o.X, &o.X, &V);
    fp_sub(&t, &V, &o.X);
    fp_mul(&t, &rr, &t);
    fp_mul(&S1, &S1, &J);
    fp_add(&S1, &S1, &S1);
    fp_sub(&o.Y, &t, &S1);
    fp_add(&t, &p->Z, &q->Z);
    fp_sqr(&t, &t);
    fp_sub(&t, &t, &Z1Z1);
    fp_sub(&t, &t, &Z2Z2);
    fp_mul(&o.Z, &t, &H);
    *r = o;
}

static void jac_neg(jac *r, const jac *p) { *r = *p; fp_neg(&r->Y, &p->Y); }

/* double-and-add, MSB first, over the integer scalar (g1p_mul.cu:18-67) */
static void jac_mul(jac *r, const jac *p, const uint64_t k[4]) {
    jac acc;
    jac_set_inf(&acc);
    for (int i = 255; i >= 0; i--) {
        jac_dbl(&acc, &acc);
        if ((k[i / 64] >> (i % 64)) & 1) jac_add(&acc, &acc, p);
    }
    *r = acc;
}

/* homogeneous projective standard-form g1p_t (x = X/Z) -> Jacobian.  Any
 * (X, Y, 0) is treated as infinity, as the reference's g1p_isInf with
 * G1P_ANYINF (g1.cuh:14, g1p_compare.cu). */
static void jac_from_g1p(jac *r, const uint64_t *g) {
    fp X, Y, Z;
    fp_from_std(&X, g);
    fp_from_std(&Y, g + 6);
    fp_from_std(&Z, g + 12);
    if (fp_is0(&Z)) { jac_set_inf(r); return; }
    fp_mul(&r->X, &X, &Z);      /* x = XZ/Z^2 */
    fp_sqr(&r->Z, &Z);
    fp_mul(&r->Y, &Y, &r->Z);   /* y = YZ^2/Z^3 */
    r->Z = Z;
}

/* Jacobian -> standard-form affine-normalised g1p_t {x, y, 1}, infinity (0,1,0). */
static void jac_to_g1p(uint64_t *g, const jac *p) {
    memset(g, 0, 144);
    if (jac_is_inf(p)) { g[6] = 1; return; }
    fp zi, zi2, zi3, x, y;
    fp_inv(&zi, &p->Z);
    fp_sqr(&zi2, &zi);
    fp_mul(&zi3, &zi2, &zi);
    fp_mul(&x, &p->X, &zi2);
    fp_mul(&y, &p->Y, &zi3);
    fp_to_std(g, &x);
    fp_to_std(g + 6, &y);
    g[12] = 1;
}

/* batch normalisation (Montgomery's trick) of n Jacobian points */
static void jac_to_g1p_batch(uint64_t *g, const jac *p, int n) {
    fp *pre = (fp *)malloc(sizeof(fp) * (n + 1));
    fp acc = FP_ONE;
    for (int i = 0; i < n; i++) {
        pre[i] = acc;
        if (!jac_is_inf(&p[i])) fp_mul(&acc, &acc, &p[i].Z);
    }
    fp inv;
    fp_inv(&inv, &acc);
    for (int i = n - 1; i >= 0; i--) {
        uint64_t *o = g + 18 * i;
        memset(o, 0, 144);
        if (jac_is_inf(&p[i])) { o[6] = 1; continue; }
        fp zi, zi2, zi3, x, y;
        fp_mul(&zi, &inv, &pre[i]);
        fp_mul(&inv, &inv, &p[i].Z);
        fp_sqr(&zi2, &zi);
        fp_mul(&zi3, &zi2, &zi);
        fp_mul(&x, &p[i].X, &zi2);
        fp_mul(&y, &p[i].Y, &zi3);
        fp_to_std(o, &x);
        fp_to_std(o + 6, &y);
        o[12] = 1;
    }
    free(pre);
}

static const uint64_t GX[6] = {0xFB3AF00ADB22C6BBULL, 0x6C55E83FF97A1AEFULL, 0xA14E3A3F171BAC58ULL,
                               0xC3688C4F9774B905ULL, 0x2695638C4FA9AC0FULL, 0x17F1D3A73197D794ULL};
static const uint64_t GY[6] = {0x0CAA232946C5E7E1ULL, 0xD03CC744A2888AE4ULL, 0x00DB18CB2C04B3EDULL,
                               0xFCF5E095D5D00AF6ULL, 0xA09E30ED741D8AE4ULL, 0x08B3F481E3AAA0F1ULL};

static void jac_gen(jac *g) {
    fp_from_std(&g->X, GX);
    fp_from_std(&g->Y, GY);
    g->Z = FP_ONE;
}

/* ------------------------------------------------------------------------- */
/* roots of unity (kzg_proofs.py:39-44)                                      */
/* ------------------------------------------------------------------------- */
static void root_of_unity(fr *w, unsigned order) {
    /* w = 5^((r-1)/order) */
    uint64_t e[4];
    memcpy(e, R_, 32);
    e[0] -= 1;
    /* divide by order (a power of two) */
    unsigned s = 0;
    while ((1u << s) < order) s++;
    for (int i = 0; i < 4; i++) {
        e[i] = (e[i] >> s) | (i < 3 && s ? (e[i + 1] << (64 - s)) : 0);
    }
    fr five;
    uint64_t f[4] = {5, 0, 0, 0};
    fr_from_std(&five, f);
    fr_pow(w, &five, e, 4);
}

/* ------------------------------------------------------------------------- */
/* FFT (fft.py:17-55): out[i] = sum_j v[j] * w^(i*j); inverse uses w^-1 and   */
/* multiplies by n^-1.  Recursive even/odd split, exactly as _fft.           */
/* ------------------------------------------------------------------------- */
static void fr_fft_rec(fr *out, const fr *in, int n, int stride, const fr *roots, int rstride) {
    if (n == 1) { out[0] = in[0]; return; }
    int h = n / 2;
    fr *L = (fr *)malloc(sizeof(fr) * n);
    fr *R = L + h;
    fr_fft_rec(L, in, h, stride * 2, roots, rstride * 2);
    fr_fft_rec(R, in + stride, h, stride * 2, roots, rstride * 2);
    for (int i = 0; i < h; i++) {
        fr t;
        fr_mul(&t, &R[i], &roots[i * rstride]);
        fr_add(&out[i], &L[i], &t);
        fr_sub(&out[i + h], &L[i], &t);
    }
    free(L);
}

static void jac_fft_rec(jac *out, const jac *in, int n, int stride, const uint64_t (*roots)[4], int rstride) {
    if (n == 1) { out[0] = in[0]; return; }
    int h = n / 2;
    jac *L = (jac *)malloc(sizeof(jac) * n);
    jac *R = L + h;
    jac_fft_rec(L, in, h, stride * 2, roots, rstride * 2);
    jac_fft_rec(R, in + stride, h, stride * 2, roots, rstride * 2);
    for (int i = 0; i < h; i++) {
        jac t, nt;
        jac_mul(&t, &R[i], roots[i * rstride]);
        jac_add(&out[i], &L[i], &t);
        jac_neg(&nt, &t);
        jac_add(&out[i + h], &L[i], &nt);
    }
    free(L);
}

/* standard-form powers of a root (integers < r) used as G1 scalars */
static void root_table_std(uint64_t (*tab)[4], int n, int inverse) {
    fr w, acc = FR_ONE;
    root_of_unity(&w, (unsigned)n);
    if (inverse) fr_inv(&w, &w);
    for (int i = 0; i < n; i++) {
        fr_to_std(tab[i], &acc);
        fr_mul(&acc, &acc, &w);
    }
}

static void fr_fft_core(fr *out, const fr *in, int n, int inverse) {
    fr *roots = (fr *)malloc(sizeof(fr) * n);
    fr w, acc = FR_ONE;
    root_of_unity(&w, (unsigned)n);
    if (inverse) fr_inv(&w, &w);
    for (int i = 0; i < n; i++) { roots[i] = acc; fr_mul(&acc, &acc, &w); }
    fr_fft_rec(out, in, n, 1, roots, 1);
    if (inverse) {
        fr ninv, nn;
        uint64_t nv[4] = {(uint64_t)n, 0, 0, 0};
        fr_from_std(&nn, nv);
        fr_inv(&ninv, &nn);
        for (int i = 0; i < n; i++) fr_mul(&out[i], &out[i], &ninv);
    }
    free(roots);
}

static void jac_fft_core(jac *out, const jac *in, int n, int inverse) {
    uint64_t (*roots)[4] = malloc(sizeof(uint64_t[4]) * n);
    root_table_std(roots, n, inverse);
    jac_fft_rec(out, in, n, 1, (const uint64_t (*)[4])roots, 1);
    if (inverse) {
        fr nn, ninv;
        uint64_t nv[4] = {(uint64_t)n, 0, 0, 0}, ns[4];
        fr_from_std(&nn, nv);
        fr_inv(&ninv, &nn);
        fr_to_std(ns, &ninv);
        for (int i = 0; i < n; i++) jac_mul(&out[i], &out[i], ns);
    }
    free(roots);
}

/* ========================================================================= */
/* exported API (ctypes).  All buffers are standard-form uint64 limbs.       */
/* ========================================================================= */

int orc_init(void) { init_consts(); return 0; }

/* Fp element-wise ops on 6-limb values; inputs may be any 384-bit value.
 * op: 0 mul, 1 sqr, 2 add, 3 sub, 4 neg, 5 inv, 6 canonicalise, 7 x2, 8 x3,
 *     9 x4, 10 x8, 11 x12.  Output canonical (< p). */
int orc_fp_op(int op, uint64_t *out, const uint64_t *a, const uint64_t *b, long count) {
    init_consts();
    for (long i = 0; i < count; i++) {
        fp x, y = {{0}}, z;
        fp_from_std(&x, a + 6 * i);
        if (b) fp_from_std(&y, b + 6 * i);
        switch (op) {
        case 0: fp_mul(&z, &x, &y); break;
        case 1: fp_sqr(&z, &x); break;
        case 2: fp_add(&z, &x, &y); break;
        case 3: fp_sub(&z, &x, &y); break;
        case 4: fp_neg(&z, &x); break;
        case 5: fp_inv(&z, &x); break;
        case 6: z = x; break;
        case 7: fp_add(&z, &x, &x); break;
        case 8: fp_add(&z, &x, &x); fp_add(&z, &z, &x); break;
        case 9: fp_add(&z, &x, &x); fp_add(&z, &z, &z); break;
        case 10: fp_add(&z, &x, &x); fp_add(&z, &z, &z); fp_add(&z, &z, &z); break;
        case 11: fp_add(&z, &x, &x); fp_add(&z, &z, &x); fp_add(&z, &z, &z); fp_add(&z, &z, &z); break;
        default: return -1;
        }
        fp_to_std(out + 6 * i, &z);
    }
    return 0;
}

/* Fr element-wise ops, same op codes as orc_fp_op (x4/x8/x12 included). */
int orc_fr_op(int op, uint64_t *out, const uint64_t *a, const uint64_t *b, long count) {
    init_consts();
    for (long i = 0; i < count; i++) {
        fr x, y = {{0}}, z;
        fr_from_std(&x, a + 4 * i);
        if (b) fr_from_std(&y, b + 4 * i);
        switch (op) {
        case 0: fr_mul(&z, &x, &y); break;
        case 1: fr_mul(&z, &x, &x); break;
        case 2: fr_add(&z, &x, &y); break;
        case 3: fr_sub(&z, &x, &y); break;
        case 4: { fr zero = {{0}}; fr_sub(&z, &zero, &x); } break;
        case 5: fr_inv(&z, &x); break;
        case 6: z = x; break;
        case 7: fr_add(&z, &x, &x); break;
        case 8: fr_add(&z, &x, &x); fr_add(&z, &z, &x); break;
        case 9: fr_add(&z, &x, &x); fr_add(&z, &z, &z); break;
        case 10: fr_add(&z, &x, &x); fr_add(&z, &z, &z); fr_add(&z, &z, &z); break;
        case 11: fr_add(&z, &x, &x); fr_add(&z, &z, &x); fr_add(&z, &z, &z); fr_add(&z, &z, &z); break;
        default: return -1;
        }
        fr_to_std(out + 4 * i, &z);
    }
    return 0;
}

/* G1 ops on g1p_t (18 limbs each).  Outputs affine-normalised {x,y,1}/(0,1,0).
 * op: 0 add(a,b), 1 dbl(a), 2 neg(a), 3 sub(a,b), 4 mul(a, scalar b[4 limbs]),
 *     5 normalise(a) */
int orc_g1_op(int op, uint64_t *out, const uint64_t *a, const uint64_t *b, long count) {
    init_consts();
    for (long i = 0; i < count; i++) {
        jac x, y, z;
        jac_from_g1p(&x, a + 18 * i);
        switch (op) {
        case 0: jac_from_g1p(&y, b + 18 * i); jac_add(&z, &x, &y); break;
        case 1: jac_dbl(&z, &x); break;
        case 2: jac_neg(&z, &x); break;
        case 3: jac_from_g1p(&y, b + 18 * i); jac_neg(&y, &y); jac_add(&z, &x, &y); break;
        case 4: jac_mul(&z, &x, b + 4 * i); break;
        case 5: z = x; break;
        default: return -1;
        }
        jac_to_g1p(out + 18 * i, &z);
    }
    return 0;
}

/* 1 if the g1p_t is on y^2 = x^3 + 4 (homogeneous: Y^2 Z = X^3 + 4 Z^3) or infinity */
int orc_g1_is_point(const uint64_t *a) {
    init_consts();
    fp X, Y, Z, l, r, t;
    fp_from_std(&X, a);
    fp_from_std(&Y, a + 6);
    fp_from_std(&Z, a + 12);
    if (fp_is0(&Z)) return fp_is0(&X) && !fp_is0(&Y);
    fp_sqr(&l, &Y);
    fp_mul(&l, &l, &Z);
    fp_sqr(&r, &X);
    fp_mul(&r, &r, &X);
    fp_sqr(&t, &Z);
    fp_mul(&t, &t, &Z);
    fp_add(&t, &t, &t);
    fp_add(&t, &t, &t);
    fp_add(&r, &r, &t);
    return fp_equal(&l, &r);
}

void orc_g1_generator(uint64_t *out) {
    init_consts();
    jac g;
    jac_gen(&g);
    jac_to_g1p(out, &g);
}

/* standard-form root of unity of the given power-of-two order */
void orc_root_of_unity(uint64_t *out, unsigned order) {
    init_consts();
    fr w;
    root_of_unity(&w, order);
    fr_to_std(out, &w);
}

/* batched Fr FFT of size n (power of two): count transforms, contiguous */
int orc_fr_fft(uint64_t *out, const uint64_t *in, int n, long count, int inverse) {
    init_consts();
    fr *a = malloc(sizeof(fr) * n), *o = malloc(sizeof(fr) * n);
    for (long c = 0; c < count; c++) {
        for (int i = 0; i < n; i++) fr_from_std(&a[i], in + 4 * ((long)c * n + i));
        fr_fft_core(o, a, n, inverse);
        for (int i = 0; i < n; i++) fr_to_std(out + 4 * ((long)c * n + i), &o[i]);
    }
    free(a);
    free(o);
    return 0;
}

/* batched G1 FFT of size n; outputs affine-normalised */
int orc_g1_fft(uint64_t *out, const uint64_t *in, int n, long count, int inverse) {
    init_consts();
    jac *a = malloc(sizeof(jac) * n), *o = malloc(sizeof(jac) * n);
    for (long c = 0; c < count; c++) {
        for (int i = 0; i < n; i++) jac_from_g1p(&a[i], in + 18 * ((long)c * n + i));
        jac_fft_core(o, a, n, inverse);
        jac_to_g1p_batch(out + 18 * (long)c * n, o, n);
    }
    free(a);
    free(o);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* seeded inputs: SplitMix64 stream; Fr values by rejection of 255-bit draws  */
/* ------------------------------------------------------------------------- */
static uint64_t splitmix_at(uint64_t seed, uint64_t i) {
    uint64_t z = seed + (i + 1) * 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

/* count uniform Fr values (< r) from the stream of `seed` */
void orc_seeded_fr(uint64_t *out, uint64_t seed, long count) {
    uint64_t j = 0;
    for (long c = 0; c < count;) {
        uint64_t v[4];
        for (int k = 0; k < 4; k++) v[k] = splitmix_at(seed, 4 * j + k);
        v[3] &= 0x7fffffffffffffffULL;
        j++;
        if (geq_n(v, R_, 4)) continue;
        memcpy(out + 4 * c, v, 32);
        c++;
    }
}

/* ------------------------------------------------------------------------- */
/* setup and FK20                                                            */
/* ------------------------------------------------------------------------- */

typedef struct {
    const uint64_t *tau; uint64_t *out; long lo, hi;
} setup_job;

static void *setup_worker(void *arg) {
    setup_job *j = arg;
    fr t, acc;
    fr_from_std(&t, j->tau);
    /* tau^lo */
    uint64_t e[4] = {(uint64_t)j->lo, 0, 0, 0};
    fr_pow(&acc, &t, e, 1);
    jac g, s;
    jac_gen(&g);
    for (long i = j->lo; i < j->hi; i++) {
        uint64_t k[4];
        fr_to_std(k, &acc);
        jac_mul(&s, &g, k);
        jac_to_g1p(j->out + 18 * i, &s);
        fr_mul(&acc, &acc, &t);
    }
    return NULL;
}

/* setup s_i = tau^i * G1 for i < count (kzg_proofs.py:22-30), affine g1p_t */
int orc_setup(uint64_t *out, const uint64_t *tau, long count, int nthreads) {
    init_consts();
    if (nthreads < 1) nthreads = 1;
    pthread_t th[64];
    setup_job jobs[64];
    if (nthreads > 64) nthreads = 64;
    for (int t = 0; t < nthreads; t++) {
        jobs[t].tau = tau; jobs[t].out = out;
        jobs[t].lo = count * t / nthreads; jobs[t].hi = count * (t + 1) / nthreads;
        pthread_create(&th[t], NULL, setup_worker, &jobs[t]);
    }
    for (int t = 0; t < nthreads; t++) pthread_join(th[t], NULL);
    return 0;
}

typedef struct { const uint64_t *setup; uint64_t *out; int n, l, i0, i1; } xext_job;

static void *xext_worker(void *arg) {
    xext_job *j = arg;
    int n = j->n, l = j->l, k = n / l;
    jac *x = malloc(sizeof(jac) * 2 * k), *o = malloc(sizeof(jac) * 2 * k);
    for (int i = j->i0; i < j->i1; i++) {
        /* x = setup[n-l-1-i :: -l] + [inf], extended with k infinities */
        int cnt = 0;
        for (int s = n - l - 1 - i; s >= 0; s -= l) jac_from_g1p(&x[cnt++], j->setup + 18 * s);
        while (cnt < 2 * k) jac_set_inf(&x[cnt++]);
        jac_fft_core(o, x, 2 * k, 0);
        jac_to_g1p_batch(j->out + 18 * (long)i * 2 * k, o, 2 * k);
    }
    free(x);
    free(o);
    return NULL;
}

/* xext_fft[l][2k] from setup (>= n-l points), FK20Py/fk20_multi_cuda.py:104-109 */
int orc_xext_fft(uint64_t *out, const uint64_t *setup, int n, int l, int nthreads) {
    init_consts();
    if (nthreads < 1) nthreads = 1;
    if (nthreads > l) nthreads = l;
    pthread_t th[64];
    xext_job jobs[64];
    for (int t = 0; t < nthreads; t++) {
        jobs[t].setup = setup; jobs[t].out = out; jobs[t].n = n; jobs[t].l = l;
        jobs[t].i0 = l * t / nthreads; jobs[t].i1 = l * (t + 1) / nthreads;
        pthread_create(&th[t], NULL, xext_worker, &jobs[t]);
    }
    for (int t = 0; t < nthreads; t++) pthread_join(th[t], NULL);
    return 0;
}

/* toeplitz coefficients of one row: tc[l][2k] (fk20_multi_cuda.py:139-146) */
void orc_toeplitz(uint64_t *tc, const uint64_t *poly, int n, int l) {
    int k = n / l;
    memset(tc, 0, 32 * (size_t)l * 2 * k);
    for (int i = 0; i < l; i++) {
        uint64_t *t = tc + 4 * (size_t)i * 2 * k;
        /* reduced_polynomial[-i-1::l] : the single element n-1-i */
        memcpy(t, poly + 4 * (size_t)(n - 1 - i), 32);
        /* [0]*(k+1) then reduced_polynomial[2l-i-1 : -l-i : l] */
        int pos = k + 2;
        for (int s = 2 * l - i - 1; s < n - l - i; s += l) memcpy(t + 4 * (size_t)pos++, poly + 4 * (size_t)s, 32);
    }
}

/* One FK20 row, FK20Py algorithm (variable-base multiply for every term).
 * Any intermediate pointer may be NULL.  tc/tc_fft: [l][2k] fr_t standard
 * canonical; hext_fft, h (2k entries, upper k = inf), h_fft: affine g1p_t. */
int orc_fk20_row(const uint64_t *poly, int n, int l, const uint64_t *xext_fft,
                 uint64_t *tc_out, uint64_t *tcfft_out, uint64_t *hext_out,
                 uint64_t *h_out, uint64_t *hfft_out) {
    init_consts();
    int k = n / l, m = 2 * k;
    uint64_t *tc = malloc(32 * (size_t)l * m);
    uint64_t *tcf = malloc(32 * (size_t)l * m);
    orc_toeplitz(tc, poly, n, l);
    orc_fr_fft(tcf, tc, m, l, 0);
    jac *hext = malloc(sizeof(jac) * m), *tmp = malloc(sizeof(jac) * m);
    for (int c = 0; c < m; c++) jac_set_inf(&hext[c]);
    for (int i = 0; i < l; i++) {
        for (int c = 0; c < m; c++) {
            jac X, t;
            jac_from_g1p(&X, xext_fft + 18 * ((size_t)i * m + c));
            jac_mul(&t, &X, tcf + 4 * ((size_t)i * m + c));
            jac_add(&hext[c], &hext[c], &t);
        }
    }
    if (hext_out) jac_to_g1p_batch(hext_out, hext, m);
    /* h = IFFT(hext_fft)[:k] ++ [inf]*k */
    jac_fft_core(tmp, hext, m, 1);
    for (int c = k; c < m; c++) jac_set_inf(&tmp[c]);
    if (h_out) jac_to_g1p_batch(h_out, tmp, m);
    jac_fft_core(hext, tmp, m, 0);
    if (hfft_out) jac_to_g1p_batch(hfft_out, hext, m);
    if (tc_out) memcpy(tc_out, tc, 32 * (size_t)l * m);
    if (tcfft_out) memcpy(tcfft_out, tcf, 32 * (size_t)l * m);
    free(tc); free(tcf); free(hext); free(tmp);
    return 0;
}

typedef struct {
    const uint64_t *poly, *xext; uint64_t *hfft; int n, l; long r0, r1;
} rows_job;

static void *rows_worker(void *arg) {
    rows_job *j = arg;
    int m = 2 * (j->n / j->l);
    for (long r = j->r0; r < j->r1; r++)
        orc_fk20_row(j->poly + 4 * (size_t)r * j->n, j->n, j->l, j->xext, NULL, NULL, NULL, NULL,
                     j->hfft + 18 * (size_t)r * m);
    return NULL;
}

/* rows x FK20 on nthreads host threads (CPU baseline) */
int orc_fk20_rows(uint64_t *h_fft, const uint64_t *poly, long rows, int n, int l,
                  const uint64_t *xext_fft, int nthreads) {
    init_consts();
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    if (nthreads > rows) nthreads = (int)rows;
    pthread_t *th = malloc(sizeof(pthread_t) * nthreads);
    rows_job *jobs = malloc(sizeof(rows_job) * nthreads);
    for (int t = 0; t < nthreads; t++) {
        jobs[t] = (rows_job){poly, xext_fft, h_fft, n, l, rows * t / nthreads, rows * (t + 1) / nthreads};
        pthread_create(&th[t], NULL, rows_worker, &jobs[t]);
    }
    for (int t = 0; t < nthreads; t++) pthread_join(th[t], NULL);
    free(th);
    free(jobs);
    return 0;
}

/* Pairing-free KZG identity (kzg_proofs.py:198-205 with tau known):
 * proof j of a row = [q_j(tau)] G1 where q_j = f div (X^l - w_2k^j) and
 * f = poly (degree < n).  Writes 2k affine points. */
int orc_kzg_direct(uint64_t *out, const uint64_t *poly, int n, int l, const uint64_t *tau,
                   int j0, int j1) {
    init_consts();
    int k = n / l, m = 2 * k;
    fr w, t, c, *f = malloc(sizeof(fr) * n), *q = malloc(sizeof(fr) * n);
    root_of_unity(&w, (unsigned)m);
    fr_from_std(&t, tau);
    for (int i = 0; i < n; i++) fr_from_std(&f[i], poly + 4 * (size_t)i);
    jac g;
    jac_gen(&g);
    for (int j = j0; j < j1; j++) {
        uint64_t e[4] = {(uint64_t)j, 0, 0, 0};
        fr_pow(&c, &w, e, 1);
        /* synthetic division by X^l - c: q[d] = f[d+l] + c*q[d+l], degrees >= n-l are 0 */
        for (int d = n - 1; d >= 0; d--) {
            if (d >= n - l) { memset(&q[d], 0, sizeof(fr)); continue; }
            fr tmp;
            if (d + l <= n - l - 1) { fr_mul(&tmp, &c, &q[d + l]); fr_add(&q[d], &f[d + l], &tmp); }
            else q[d] = f[d + l];
        }
        /* evaluate q at tau (Horner) */
        fr acc = {{0}};
        for (int d = n - l - 1; d >= 0; d--) { fr_mul(&acc, &acc, &t); fr_add(&acc, &acc, &q[d]); }
        uint64_t ks[4];
        fr_to_std(ks, &acc);
        jac pt;
        jac_mul(&pt, &g, ks);
        jac_to_g1p(out + 18 * (size_t)(j - j0), &pt);
    }
    free(f);
    free(q);
    return 0;
}
