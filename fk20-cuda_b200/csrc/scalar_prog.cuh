// scalar_prog.cuh -- fixed-scalar G1 multiplication programs (GLV + wNAF).
//
// Every G1 FFT butterfly multiplies a data-dependent point by a FIXED scalar,
// a power of the 512th root of unity w = 5^((r-1)/512) (the table fr_roots,
// fr_roots.cu:17-533; the reference runs a 256-bit double-and-add per twiddle,
// g1p_mul.cu:18-67).  Here each fixed scalar k is decomposed once on the host
// with the GLV endomorphism of BLS12-381 G1: k = k1 + k2*lambda (mod r) with
// lambda = z^2 - 1 ~ 2^128, r = lambda^2 + lambda + 1, so k2 = k div lambda and
// k1 = k mod lambda are both < 2^128, and [k]P = [k1]P + [k2]phi(P) with
// phi(x, y) = (beta x, y).  k1 and k2 are recoded in width-4 NAF (digits 0,
// +-1, +-3, +-5, +-7; nonzero digits at least 4 apart) and processed jointly
// over the precomputed P, 3P, 5P, 7P and their images under phi, which differ
// only in x (beta x): ~124 doublings and ~49 additions instead of ~254 and
// ~128.  Of k and r - k the cheaper one is encoded (and the result negated).
// The result equals [k]P for every P in the order-r subgroup -- all FK20 data.
//
// Program layout (PROG_WORDS uint32 words):
//   word 0      : bits 0-7 top digit position, bit 8 = scalar is 0,
//                 bit 9 = scalar is +-1, bit 10 = negate the result
//   words 1..34 : one byte per digit position p (word 1 + p/4, byte p%4):
//                 bits 0-3 the k1 digit, bits 4-7 the k2 digit, each coded as
//                 bit0 nonzero, bit1 negative, bits 2-3 (|digit| - 1) / 2
// A warp runs one program for 32 independent points, so every branch in the
// executor is warp-uniform.
#pragma once
#include "g1.cuh"

namespace fk {

constexpr int PROG_POSITIONS = 136;
constexpr int PROG_WORDS = 1 + PROG_POSITIONS / 4;
constexpr int PROG_SLOTS = 4;                         // P, 3P, 5P, 7P
constexpr int PROG_SLOT_WORDS = 36 * PROG_SLOTS + 12;  // (x', y', beta x') of each point, then u

// The executor's scratch: for each thread PROG_SLOT_WORDS 32-bit words at
// base[0], base[stride], ...  While P, 3P, 5P, 7P are formed, point i is
// projective (X, Y, Z) at word 36 i.  The main loop then reads point i as
// (x', y', beta x') at words 36 i, 36 i + 12, 36 i + 24 -- affine coordinates
// on an isomorphic curve, see g1_mul_prog -- and the scale factor u at word
// 144.  Addresses are formed when used, so the scratch costs one pointer of
// registers.
struct ProgSlots {
    uint32_t *base;
    int stride;
    FK_HD StridedPoint pt(int i) const { return StridedPoint{base + 36 * i * stride, stride}; }
    FK_HD StridedPoint operator[](int i) const { return pt(i); }
    FK_HD uint32_t *word(int w) const { return base + w * stride; }
};

FK_HD void slot_put(uint32_t *dst, int stride, const Fp &f) {
#pragma unroll
    for (int k = 0; k < 12; k++) dst[k * stride] = f.w[k];
}
FK_HD void slot_get(Fp &f, const uint32_t *src, int stride) {
#pragma unroll
    for (int k = 0; k < 12; k++) f.w[k] = src[k * stride];
}

// Q = point i of the main loop's table or its image phi(Q) = (beta x', y'):
// x read from one of two places, y shared
struct SlotQ {
    const uint32_t *x, *y;
    int stride;
    FK_HD void get(int c, Fp &f) const { slot_get(f, c == 0 ? x : y, stride); }
};

// acc = [k] P for the program of k (P in the prime-order subgroup, or P =
// infinity), P read from point 0 of the slots, result in homogeneous
// projective coordinates.
//
// 1. P to Jacobian coordinates; 2P with P moved onto its Z (the doubling
//    gives that for free), then 3P, 5P, 7P by co-Z additions of 2P (Meloni),
//    each of which moves 2P onto the new Z; P, 3P and 5P are then brought
//    onto the Z of 7P, u, by their steps' factors.  The four points share
//    Z = u: their (x, y) are affine coordinates on the isomorphic curve
//    E': y^2 = x^3 + b u^6, which (x, y) -> (u^2 x, u^3 y) maps E to, and
//    phi commutes with the isomorphism, so phi of a table point is
//    (beta x', y') there too.  No exceptional case for points of order r
//    (2P != +-P, 3P != +-2P, 5P != +-2P).
// 2. The digits run on E' with a Jacobian accumulator: doublings of 7 and
//    mixed additions of 11 Fp products (instead of 8 and 12 for the complete
//    projective formulas), as neither formula uses b.  The mixed addition is
//    not complete; for points of order r the accumulator never equals the
//    added point or its negative, nor infinity (the program's partial sums,
//    checked on the CPU for every program the library builds).
// 3. Back to E: Jacobian (X, Y, Z u), i.e. homogeneous (X Z', Y, Z'^3) with
//    Z' = Z u.  P = infinity (u = 0) makes every value above meaningless;
//    the lane's flag then selects infinity.
template <class ProgPtr>
FK_HD void g1_mul_prog(G1P &acc, const ProgSlots &slot, ProgPtr prog) {
    const uint32_t hdr = prog[0];
    if (hdr & 0x100u) { g1_set_inf(acc); return; }
    const bool negate = (hdr & 0x400u) != 0;
    if (hdr & 0x200u) {
        slot.pt(0).load(acc);
        if (negate) f_neg(acc.y, acc.y);
        return;
    }
    const int st = slot.stride;
    bool inf;
    {
        // P: homogeneous (X, Y, Z) -> Jacobian (X Z, Y Z^2, Z)
        G1P p;
        slot.pt(0).load(p);
        inf = f_is_zero(p.z);
        G1J a, b;
        Fp t;
        fp_sqr(t, p.z);
        fp_mul(b.x, p.x, p.z);
        fp_mul(b.y, p.y, t);
        b.z = p.z;
        // a = 2P, b = P on the Z of 2P; then b = 3P, 5P, 7P by co-Z additions
        // of a, each of which moves a (2P) onto the new Z.  Point i keeps its
        // (x, y); the factor e of its step waits in its beta x place.
        g1j_dblu(a, b, b);
        slot_put(slot.word(0), st, b.x);
        slot_put(slot.word(12), st, b.y);
#pragma unroll 1
        for (int i = 1; i < PROG_SLOTS; i++) {
            g1j_zaddu(b, a, b, t);
            slot_put(slot.word(36 * i), st, b.x);
            slot_put(slot.word(36 * i + 12), st, b.y);
            slot_put(slot.word(36 * i + 24), st, t);
        }
        slot_put(slot.word(144), st, b.z);  // u: the Z of 7P
    }
    {
        // onto the Z of 7P: 5P by e3, 3P by e2 e3, P by e1 e2 e3
        // ((x, y) -> (f^2 x, f^3 y)); then beta x' of every point
        Fp f, g, f2, c;
        slot_get(f, slot.word(36 * 3 + 24), st);
#pragma unroll 1
        for (int i = PROG_SLOTS - 2; i >= 0; i--) {
            if (i < PROG_SLOTS - 2) {
                slot_get(g, slot.word(36 * (i + 1) + 24), st);
                fp_mul(f, f, g);
            }
            uint32_t *q = slot.word(36 * i);
            fp_sqr(f2, f);
            slot_get(c, q, st);
            fp_mul(c, c, f2);
            slot_put(q, st, c);
            fp_mul(f2, f2, f);
            slot_get(c, q + 12 * st, st);
            fp_mul(c, c, f2);
            slot_put(q + 12 * st, st, c);
        }
#pragma unroll
        for (int i = 0; i < 12; i++) f.w[i] = beta_mont(i);
#pragma unroll 1
        for (int i = 0; i < PROG_SLOTS; i++) {
            uint32_t *q = slot.word(36 * i);
            slot_get(c, q, st);
            fp_mul(c, c, f);
            slot_put(q + 24 * st, st, c);  // beta x'
        }
    }
    G1J j;
    const int top = (int)(hdr & 0xffu);
    bool started = false;
    for (int pos = top; pos >= 0; pos--) {
        if (started) g1j_dbl(j, j);
        const uint32_t byte = (prog[1 + (pos >> 2)] >> ((pos & 3) * 8)) & 0xffu;
        for (int h = 0; h < 2; h++) {
            const uint32_t d = (byte >> (4 * h)) & 15u;
            if (d & 1u) {
                const uint32_t *pt = slot.word(36 * (int)(d >> 2));
                const SlotQ q{h ? pt + 24 * st : pt, pt + 12 * st, st};
                if (started) {
                    g1j_madd(j, j, q, (d & 2u) != 0);
                } else {
                    q.get(0, j.x);
                    q.get(1, j.y);
                    if (d & 2u) f_neg(j.y, j.y);
                    f_set_one(j.z);
                }
                started = true;
            }
        }
    }
    if (negate) f_neg(j.y, j.y);
    {
        Fp u, t;
        slot_get(u, slot.word(144), st);
        fp_mul(j.z, j.z, u);  // Z' = Z u
        fp_mul(acc.x, j.x, j.z);
        fp_sqr(t, j.z);
        fp_mul(acc.z, t, j.z);
        acc.y = j.y;
    }
    if (inf) g1_set_inf(acc);
}

// register-only convenience form (setup-time and element-wise kernels): a
// local scratch array stands in for the slots
template <class ProgPtr>
FK_HD void g1_mul_prog(G1P &R, const G1P &P, ProgPtr prog) {
    uint32_t mem[PROG_SLOT_WORDS];
    const ProgSlots slot{mem, 1};
    slot.pt(0).put(P);
    g1_mul_prog(R, slot, prog);
}

// ---------------------------------------------------------------- host side (host-only functions)
// little-endian 64-bit word big integers, just enough for the decomposition
namespace host {

inline int cmp_words(const uint64_t *a, const uint64_t *b, int n) {
    for (int i = n - 1; i >= 0; i--)
        if (a[i] != b[i]) return a[i] > b[i] ? 1 : -1;
    return 0;
}

// q = a div d, rem = a mod d for 256-bit a and d (shift-subtract)
inline void divmod256(uint64_t q[4], uint64_t rem[4], const uint64_t a[4], const uint64_t d[4]) {
    uint64_t r[4] = {0, 0, 0, 0};
    for (int i = 0; i < 4; i++) q[i] = 0;
    for (int bit = 255; bit >= 0; bit--) {
        for (int i = 3; i > 0; i--) r[i] = (r[i] << 1) | (r[i - 1] >> 63);
        r[0] = (r[0] << 1) | ((a[bit / 64] >> (bit % 64)) & 1);
        if (cmp_words(r, d, 4) >= 0) {
            unsigned __int128 br = 0;
            for (int i = 0; i < 4; i++) {
                unsigned __int128 t = (unsigned __int128)r[i] - d[i] - br;
                r[i] = (uint64_t)t;
                br = (t >> 64) ? 1 : 0;
            }
            q[bit / 64] |= 1ull << (bit % 64);
        }
    }
    for (int i = 0; i < 4; i++) rem[i] = r[i];
}

// width-4 NAF digits (0, +-1, +-3, +-5, +-7) of k < 2^128 into
// d[0..PROG_POSITIONS); returns the top position or -1
inline int wnaf4(int8_t *d, unsigned __int128 k) {
    int top = -1;
    for (int i = 0; i < PROG_POSITIONS; i++) d[i] = 0;
    for (int i = 0; k != 0; i++) {
        if (k & 1) {
            int v = (int)(k & 15);
            if (v >= 8) v -= 16;
            d[i] = (int8_t)v;
            if (v > 0) k -= (unsigned)v; else k += (unsigned)(-v);
            top = i;
        }
        k >>= 1;
    }
    return top;
}

inline uint32_t digit_code(int v) {
    if (v == 0) return 0;
    const int m = v < 0 ? -v : v;
    return 1u | (v < 0 ? 2u : 0u) | ((uint32_t)((m - 1) / 2) << 2);
}

// program for a standard-form scalar k < r (4 x 64-bit words), no sign choice
inline void make_program_raw(uint32_t prog[PROG_WORDS], const uint64_t k[4]) {
    static const uint64_t LAMBDA[4] = {0x00000000ffffffffull, 0xac45a4010001a402ull, 0, 0};
    for (int i = 0; i < PROG_WORDS; i++) prog[i] = 0;
    const bool zero = (k[0] | k[1] | k[2] | k[3]) == 0;
    const bool one = k[0] == 1 && (k[1] | k[2] | k[3]) == 0;
    if (zero) { prog[0] = 0x100u; return; }
    if (one) { prog[0] = 0x200u; return; }
    uint64_t q[4], rem[4];
    divmod256(q, rem, k, LAMBDA);
    unsigned __int128 k1 = ((unsigned __int128)rem[1] << 64) | rem[0];
    unsigned __int128 k2 = ((unsigned __int128)q[1] << 64) | q[0];
    int8_t d1[PROG_POSITIONS], d2[PROG_POSITIONS];
    int t1 = wnaf4(d1, k1), t2 = wnaf4(d2, k2);
    int top = t1 > t2 ? t1 : t2;
    prog[0] = (uint32_t)top;
    for (int p = 0; p <= top; p++) {
        const uint32_t byte = digit_code(d1[p]) | (digit_code(d2[p]) << 4);
        prog[1 + (p >> 2)] |= byte << ((p & 3) * 8);
    }
}

// algorithmic cost of a program in doublings and additions (the 3P, 5P, 7P
// precompute included: 1 doubling + 3 additions; the four phi products are not)
inline void program_cost(const uint32_t prog[PROG_WORDS], int *dbl, int *add) {
    *dbl = *add = 0;
    if (prog[0] & 0x300u) return;
    int top = (int)(prog[0] & 0xff);
    bool started = false;
    *dbl = 1;
    *add = PROG_SLOTS - 1;
    for (int p = top; p >= 0; p--) {
        if (started) (*dbl)++;
        const uint32_t byte = (prog[1 + (p >> 2)] >> ((p & 3) * 8)) & 0xff;
        for (int h = 0; h < 2; h++) {
            if ((byte >> (4 * h)) & 1) {
                if (started) (*add)++;
                started = true;
            }
        }
    }
}

// program for k: the cheaper of k and (r - k) followed by a negation
inline void make_program(uint32_t prog[PROG_WORDS], const uint64_t k[4]) {
    static const uint64_t R[4] = {0xffffffff00000001ull, 0x53bda402fffe5bfeull, 0x3339d80809a1d805ull,
                                  0x73eda753299d7d48ull};
    make_program_raw(prog, k);
    if ((k[0] | k[1] | k[2] | k[3]) == 0) return;
    uint64_t nk[4];
    unsigned __int128 br = 0;
    for (int i = 0; i < 4; i++) {
        unsigned __int128 t = (unsigned __int128)R[i] - k[i] - br;
        nk[i] = (uint64_t)t;
        br = (t >> 64) ? 1 : 0;
    }
    uint32_t alt[PROG_WORDS];
    make_program_raw(alt, nk);
    int d0, a0, d1, a1;
    program_cost(prog, &d0, &a0);
    program_cost(alt, &d1, &a1);
    if (7 * d1 + 11 * a1 < 7 * d0 + 11 * a0) {
        alt[0] |= 0x400u;
        for (int i = 0; i < PROG_WORDS; i++) prog[i] = alt[i];
    }
}

}  // namespace host

}  // namespace fk
