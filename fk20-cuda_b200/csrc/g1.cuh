// g1.cuh -- BLS12-381 G1 (y^2 = x^3 + 4 over Fp) in homogeneous projective
// coordinates (x = X/Z, y = Y/Z), the reference's convention (g1.cuh:20-29),
// with the complete addition laws of Renes, Costello and Batina (eprint
// 2015/1060): Algorithm 7 (addition), 8 (mixed addition) and 9 (doubling) for
// a = 0, b3 = 3*b = 12.  Complete means no exceptional inputs: P + P, P + (-P)
// and the point at infinity (0 : Y : 0) all go through the same straight-line
// code, so warps never diverge on point values.  Coordinates are Montgomery
// Fp elements (field.cuh).
#pragma once
#include "field.cuh"

namespace fk {

// Fp products of the curve formulas.  A translation unit that defines
// FK_FP_MUL_OUTLINE gets one out-of-line copy of the ~700-instruction product
// that every call site shares (operands and result pass in registers): loops
// over point operations then fit the instruction cache instead of streaming
// hundreds of KB of inlined code.  Otherwise the product is inlined.
#if defined(__CUDACC__) && defined(FK_FP_MUL_OUTLINE)
static __device__ __noinline__ Fp fp_mul_outline(Fp a, Fp b) {
    Fp r;
    f_mul(r, a, b);
    return r;
}
#endif

FK_HD void fp_mul(Fp &r, const Fp &a, const Fp &b) {
#if defined(__CUDA_ARCH__) && defined(FK_FP_MUL_OUTLINE)
    r = fp_mul_outline(a, b);
#else
    f_mul(r, a, b);
#endif
}

// Squares take the triangular Montgomery square (field.cuh: 78 + 156 limb
// products instead of 144 + 156), out of line in the same translation units.
#if defined(__CUDACC__) && defined(FK_FP_MUL_OUTLINE)
static __device__ __noinline__ Fp fp_sqr_outline(Fp a) {
    Fp r;
    f_sqr(r, a);
    return r;
}
#endif

FK_HD void fp_sqr(Fp &r, const Fp &a) {
#if defined(__CUDA_ARCH__) && defined(FK_FP_MUL_OUTLINE)
    r = fp_sqr_outline(a);
#else
    f_sqr(r, a);
#endif
}

struct G1P {
    Fp x, y, z;
};
struct G1A {
    Fp x, y;
};

FK_HD void g1_set_inf(G1P &p) {
    f_set_zero(p.x);
    f_set_one(p.y);
    f_set_zero(p.z);
}

FK_HD bool g1_is_inf(const G1P &p) { return f_is_zero(p.z); }

FK_HD void g1_neg(G1P &r, const G1P &p) {
    r.x = p.x;
    f_neg(r.y, p.y);
    r.z = p.z;
}

// Q accessor for a point held in registers
struct RegPoint {
    const G1P &p;
    FK_HD void get(int c, Fp &f) const { f = c == 0 ? p.x : c == 1 ? p.y : p.z; }
};

// Q accessor for a point stored word-strided (word k at base[k * stride]),
// e.g. one thread's slot in a conflict-free shared-memory array
struct StridedPoint {
    uint32_t *base;
    int stride;
    FK_HD void get(int c, Fp &f) const {
#pragma unroll
        for (int k = 0; k < 12; k++) f.w[k] = base[(12 * c + k) * stride];
    }
    FK_HD void put(const G1P &p) const {
#pragma unroll
        for (int k = 0; k < 12; k++) {
            base[k * stride] = p.x.w[k];
            base[(12 + k) * stride] = p.y.w[k];
            base[(24 + k) * stride] = p.z.w[k];
        }
    }
    FK_HD void load(G1P &p) const {
        get(0, p.x);
        get(1, p.y);
        get(2, p.z);
    }
};

// R = P + (negQ ? -Q : Q), Algorithm 7 with Q read through an accessor as
// needed (keeps Q out of registers) and the sign folded into the two places
// Y2 enters: t1 = Y1*Y2 and the sums X2+Y2, Y2+Z2.
template <class QT>
FK_HD void g1_add_q(G1P &R, const G1P &P, const QT &Q, bool negQ) {
    Fp t0, t1, t2, t3, t4, X3, Y3, Z3, q;
    Q.get(0, q);
    fp_mul(t0, P.x, q);
    Q.get(1, q);
    fp_mul(t1, P.y, q);
    if (negQ) f_neg(t1, t1);
    Q.get(2, q);
    fp_mul(t2, P.z, q);
    f_add(t3, P.x, P.y);
    Q.get(0, q);
    Q.get(1, t4);
    if (negQ) f_sub(t4, q, t4); else f_add(t4, q, t4);
    fp_mul(t3, t3, t4);
    f_add(t4, t0, t1);
    f_sub(t3, t3, t4);
    f_add(t4, P.y, P.z);
    Q.get(2, q);
    Q.get(1, X3);
    if (negQ) f_sub(X3, q, X3); else f_add(X3, X3, q);
    fp_mul(t4, t4, X3);
    f_add(X3, t1, t2);
    f_sub(t4, t4, X3);
    f_add(X3, P.x, P.z);
    Q.get(0, q);
    Q.get(2, Y3);
    f_add(Y3, q, Y3);
    fp_mul(X3, X3, Y3);
    f_add(Y3, t0, t2);
    f_sub(Y3, X3, Y3);
    f_add(X3, t0, t0);
    f_add(t0, X3, t0);
    f_mul12(t2, t2);
    f_add(Z3, t1, t2);
    f_sub(t1, t1, t2);
    f_mul12(Y3, Y3);
    fp_mul(X3, t4, Y3);
    fp_mul(t2, t3, t1);
    f_sub(X3, t2, X3);
    fp_mul(Y3, Y3, t0);
    fp_mul(t1, t1, Z3);
    f_add(Y3, t1, Y3);
    fp_mul(t0, t0, t3);
    fp_mul(Z3, Z3, t4);
    f_add(Z3, Z3, t0);
    R.x = X3;
    R.y = Y3;
    R.z = Z3;
}

// R = P + Q (RCB Algorithm 7, 12 M + 2 m_3b)
FK_HD void g1_add(G1P &R, const G1P &P, const G1P &Q) { g1_add_q(R, P, RegPoint{Q}, false); }

// R = P + (qx, qy) with Q affine and not infinity (RCB Algorithm 8, 11 M + 2 m_3b)
FK_HD void g1_madd(G1P &R, const G1P &P, const Fp &qx, const Fp &qy) {
    Fp t0, t1, t2, t3, t4, X3, Y3, Z3;
    fp_mul(t0, P.x, qx);
    fp_mul(t1, P.y, qy);
    f_add(t3, qx, qy);
    f_add(t4, P.x, P.y);
    fp_mul(t3, t3, t4);
    f_add(t4, t0, t1);
    f_sub(t3, t3, t4);
    fp_mul(t4, qy, P.z);
    f_add(t4, t4, P.y);
    fp_mul(Y3, qx, P.z);
    f_add(Y3, Y3, P.x);
    f_add(X3, t0, t0);
    f_add(t0, X3, t0);
    f_mul12(t2, P.z);
    f_add(Z3, t1, t2);
    f_sub(t1, t1, t2);
    f_mul12(Y3, Y3);
    fp_mul(X3, t4, Y3);
    fp_mul(t2, t3, t1);
    f_sub(X3, t2, X3);
    fp_mul(Y3, Y3, t0);
    fp_mul(t1, t1, Z3);
    f_add(Y3, t1, Y3);
    fp_mul(t0, t0, t3);
    fp_mul(Z3, Z3, t4);
    f_add(Z3, Z3, t0);
    R.x = X3;
    R.y = Y3;
    R.z = Z3;
}

// R = 2P (RCB Algorithm 9, 6 M + 2 S + 1 m_3b), with the products reordered
// so that the inputs die early: at most 6 field temporaries are live at once
// (the listed order keeps 8), which matters when the products are
// out-of-line calls and every live value holds a register across them.
FK_HD void g1_dbl(G1P &R, const G1P &P) {
    Fp t0, t1, t2, t3, X3, Y3, Z3;
    fp_sqr(t0, P.y);         // Y^2
    fp_mul(t3, P.x, P.y);    // XY
    fp_mul(t1, P.y, P.z);    // YZ
    fp_sqr(t2, P.z);         // Z^2
    f_mul12(t2, t2);         // b3 Z^2
    f_add(Z3, t0, t0);
    f_add(Z3, Z3, Z3);
    f_add(Z3, Z3, Z3);       // 8 Y^2
    fp_mul(X3, t2, Z3);
    fp_mul(Z3, t1, Z3);      // 8 Y^3 Z
    f_add(Y3, t0, t2);
    f_add(t1, t2, t2);
    f_add(t2, t1, t2);       // 3 b3 Z^2
    f_sub(t0, t0, t2);
    fp_mul(Y3, t0, Y3);
    f_add(Y3, X3, Y3);
    fp_mul(X3, t0, t3);
    f_add(X3, X3, X3);
    R.x = X3;
    R.y = Y3;
    R.z = Z3;
}

// ---------------------------------------------------------------- Jacobian, a = 0
// Jacobian coordinates (x = X/Z^2, y = Y/Z^3), used inside the fixed-scalar
// programs (scalar_prog.cuh).  The formulas below do not involve the curve
// constant b, so they hold on every curve y^2 = x^3 + b' -- in particular on
// the isomorphic curve b' = b u^6 on which a program's precomputed points are
// affine.
struct G1J {
    Fp x, y, z;
};

// R = 2P (2 M + 5 S, "dbl-2009-l" of the Explicit-Formulas Database); R may
// alias P.  Infinity (Z = 0) stays infinity; no other exceptional input on a
// curve without points of order 2.
FK_HD void g1j_dbl(G1J &R, const G1J &P) {
    Fp A, B, C, D, t;
    fp_mul(t, P.y, P.z);  // Y Z
    fp_sqr(B, P.y);       // B = Y^2
    fp_sqr(A, P.x);       // A = X^2
    fp_sqr(C, B);         // C = Y^4
    f_add(D, P.x, B);
    fp_sqr(D, D);
    f_sub(D, D, A);
    f_sub(D, D, C);
    f_add(D, D, D);       // D = 2 ((X + B)^2 - A - C) = 4 X Y^2
    f_add(R.z, t, t);     // Z3 = 2 Y Z
    f_add(t, A, A);
    f_add(A, t, A);       // E = 3 A
    fp_sqr(t, A);         // F = E^2
    f_sub(t, t, D);
    f_sub(R.x, t, D);     // X3 = F - 2 D
    f_sub(t, D, R.x);
    fp_mul(t, A, t);      // E (D - X3)
    f_add(C, C, C);
    f_add(C, C, C);
    f_add(C, C, C);       // 8 C
    f_sub(R.y, t, C);     // Y3 = E (D - X3) - 8 C
}

// R = 2P and S = P moved onto the Z of R: S = (X (2Y)^2, Y (2Y)^3, 2 Y Z),
// which dbl-2009-l computes anyway as (D, 8 C, Z3) ("DBLU" of the co-Z
// literature); 2 M + 5 S.  R and S may alias P.
FK_HD void g1j_dblu(G1J &R, G1J &S, const G1J &P) {
    Fp A, B, C, D, t, y3;
    fp_mul(t, P.y, P.z);  // Y Z
    fp_sqr(B, P.y);       // B = Y^2
    fp_sqr(A, P.x);       // A = X^2
    fp_sqr(C, B);         // C = Y^4
    f_add(D, P.x, B);
    fp_sqr(D, D);
    f_sub(D, D, A);
    f_sub(D, D, C);
    f_add(D, D, D);       // D = 4 X Y^2
    f_add(t, t, t);       // Z3 = 2 Y Z
    f_add(B, A, A);
    f_add(A, B, A);       // E = 3 A
    fp_sqr(B, A);         // F = E^2
    f_sub(B, B, D);
    f_sub(B, B, D);       // X3 = F - 2 D
    f_add(C, C, C);
    f_add(C, C, C);
    f_add(C, C, C);       // 8 C
    f_sub(y3, D, B);
    fp_mul(y3, A, y3);
    f_sub(y3, y3, C);     // Y3 = E (D - X3) - 8 C
    R.x = B;
    R.y = y3;
    R.z = t;
    S.x = D;
    S.y = C;
    S.z = t;
}

// Co-Z addition (Meloni, "ZADDU"): A = (X1, Y1, Z) and B = (X2, Y2, Z) share
// Z, A != +-B.  R = A + B with Z3 = Z e, e = X2 - X1, and A is moved onto
// that Z: A = (X1 e^2, Y1 e^3, Z e); e is returned.  5 M + 2 S.  R may alias
// B (not A).
FK_HD void g1j_zaddu(G1J &R, G1J &A, const G1J &B, Fp &e) {
    Fp c, w1, w2, d, h, x3;
    f_sub(e, B.x, A.x);    // e = X2 - X1
    fp_sqr(c, e);          // e^2
    fp_mul(w1, A.x, c);    // W1 = X1 e^2
    fp_mul(w2, B.x, c);    // W2 = X2 e^2
    f_sub(h, B.y, A.y);    // Y2 - Y1
    fp_sqr(d, h);          // (Y2 - Y1)^2
    f_sub(c, w2, w1);      // e^3
    fp_mul(c, A.y, c);     // Y1 e^3
    f_sub(x3, d, w1);
    f_sub(x3, x3, w2);     // X3 = (Y2 - Y1)^2 - W1 - W2
    f_sub(d, w1, x3);
    fp_mul(d, h, d);
    f_sub(R.y, d, c);      // Y3 = (Y2 - Y1) (W1 - X3) - Y1 e^3
    fp_mul(A.z, A.z, e);   // Z3 = Z e
    R.x = x3;
    R.z = A.z;
    A.x = w1;
    A.y = c;
}

// R = P + (negQ ? -Q : Q) with Q = (x, y) affine, read through an accessor
// (get(0) = x, get(1) = y); 8 M + 3 S ("madd-2007-bl" with Z3 = 2 Z1 H).
// NOT complete: P = +-Q (H = 0) and P = infinity give wrong results.  The
// fixed-scalar programs never meet either for points of order r (a CPU test
// checks every program's partial sums); R may alias P.
template <class QT>
FK_HD void g1j_madd(G1J &R, const G1J &P, const QT &Q, bool negQ) {
    Fp zz, u, s, h, t, j;
    fp_sqr(zz, P.z);       // Z1^2
    Q.get(0, t);
    fp_mul(u, t, zz);      // U2 = X2 Z1^2
    fp_mul(s, P.z, zz);    // Z1^3
    Q.get(1, t);
    fp_mul(s, t, s);       // S2 = Y2 Z1^3
    if (negQ) f_neg(s, s);
    f_sub(h, u, P.x);      // H = U2 - X1
    fp_mul(t, P.z, h);
    f_add(R.z, t, t);      // Z3 = 2 Z1 H
    fp_sqr(t, h);
    f_add(t, t, t);
    f_add(t, t, t);        // I = 4 H^2
    fp_mul(j, h, t);       // J = H I
    fp_mul(u, P.x, t);     // V = X1 I
    f_sub(s, s, P.y);
    f_add(s, s, s);        // r = 2 (S2 - Y1)
    fp_mul(t, P.y, j);     // Y1 J
    fp_sqr(h, s);
    f_sub(h, h, j);
    f_sub(h, h, u);
    f_sub(R.x, h, u);      // X3 = r^2 - J - 2 V
    f_sub(u, u, R.x);
    fp_mul(u, s, u);       // r (V - X3)
    f_add(t, t, t);
    f_sub(R.y, u, t);      // Y3 = r (V - X3) - 2 Y1 J
}

// affine normalisation in Montgomery form: (x, y, 1) or infinity (0, 1, 0)
FK_HD void g1_normalize(G1P &p) {
    if (f_is_zero(p.z)) {
        g1_set_inf(p);
        return;
    }
    Fp zi;
    f_inv(zi, p.z);
    f_mul(p.x, p.x, zi);
    f_mul(p.y, p.y, zi);
    f_set_one(p.z);
}

// GLV endomorphism phi(x, y) = (beta x, y) = [lambda] P on G1, with
// lambda = z^2 - 1 (z = -0xd201000000010000) and beta the cube root of unity
// in Fp below (Montgomery form).  r = lambda^2 + lambda + 1.
FK_HD constexpr uint32_t beta_mont(int i) {
    return i == 0 ? 0x8671f071u : i == 1 ? 0xcd03c9e4u : i == 2 ? 0x1fcda5d2u : i == 3 ? 0x5dab2246u
         : i == 4 ? 0xd3851b95u : i == 5 ? 0x587042afu : i == 6 ? 0x01bacb9eu : i == 7 ? 0x8eb60ebeu
         : i == 8 ? 0x83d050d2u : i == 9 ? 0x03f97d6eu : i == 10 ? 0x54638741u : 0x18f02065u;
}

FK_HD void g1_phi(G1P &R, const G1P &P) {
    Fp beta;
#pragma unroll
    for (int i = 0; i < 12; i++) beta.w[i] = beta_mont(i);
    fp_mul(R.x, P.x, beta);
    R.y = P.y;
    R.z = P.z;
}

}  // namespace fk
