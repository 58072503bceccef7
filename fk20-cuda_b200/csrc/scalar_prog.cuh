// scalar_prog.cuh -- fixed-scalar G1 multiplication programs (GLV + NAF).
//
// Every G1 FFT butterfly multiplies a data-dependent point by a FIXED scalar,
// a power of the 512th root of unity w = 5^((r-1)/512) (the table fr_roots,
// fr_roots.cu:17-533; the reference runs a 256-bit double-and-add per twiddle,
// g1p_mul.cu:18-67).  Here each fixed scalar k is decomposed once on the host
// with the GLV endomorphism of BLS12-381 G1: k = k1 + k2*lambda (mod r) with
// lambda = z^2 - 1 ~ 2^128, r = lambda^2 + lambda + 1, so k2 = k div lambda and
// k1 = k mod lambda are both < 2^128, and [k]P = [k1]P + [k2]phi(P) with
// phi(x, y) = (beta x, y).  k1 and k2 are recoded in NAF and interleaved:
// ~128 doublings and ~86 additions instead of ~254 and ~128.  The result is
// the same group element for every P in the order-r subgroup (all FK20 data).
//
// Program layout (PROG_WORDS uint32 words):
//   word 0       : bits 0-7 top digit position (0..135), bit 8 = scalar is 0,
//                  bit 9 = scalar is +-1, bit 10 = negate the result (the
//                  program encodes r - k when that is cheaper)
//   words 1..17  : 4 bits per digit position p (word 1 + p/8, nibble p%8):
//                  bit0 k1-digit nonzero, bit1 k1-digit negative,
//                  bit2 k2-digit nonzero, bit3 k2-digit negative
// Warps run one program for 32 independent points, so every branch in the
// executor is warp-uniform.
#pragma once
#include "g1.cuh"

namespace fk {

constexpr int PROG_WORDS = 18;
constexpr int PROG_POSITIONS = 8 * (PROG_WORDS - 1);

// acc = [k] P for the program of k (P in the prime-order subgroup).  P is
// read from the strided slot sP; phi(P) is written to sPhi first.  Only the
// accumulator lives in registers.
template <class ProgPtr>
FK_HD void g1_mul_prog(G1P &acc, const StridedPoint &sP, const StridedPoint &sPhi, ProgPtr prog) {
    const uint32_t hdr = prog[0];
    if (hdr & 0x100u) { g1_set_inf(acc); return; }
    const bool negate = (hdr & 0x400u) != 0;
    if (hdr & 0x200u) {
        sP.load(acc);
        if (negate) f_neg(acc.y, acc.y);
        return;
    }
    {
        G1P phi;
        sP.get(0, phi.x);
        Fp beta;
#pragma unroll
        for (int i = 0; i < 12; i++) beta.w[i] = beta_mont(i);
        f_mul(phi.x, phi.x, beta);
        sP.get(1, phi.y);
        sP.get(2, phi.z);
        sPhi.put(phi);
    }
    const int top = (int)(hdr & 0xffu);
    bool started = false;
    for (int pos = top; pos >= 0; pos--) {
        if (started) g1_dbl(acc, acc);
        const uint32_t nib = (prog[1 + (pos >> 3)] >> ((pos & 7) * 4)) & 0xfu;
        if (nib & 1u) {
            if (started) {
                g1_add_q(acc, acc, sP, (nib & 2u) != 0);
            } else {
                sP.load(acc);
                if (nib & 2u) f_neg(acc.y, acc.y);
            }
            started = true;
        }
        if (nib & 4u) {
            if (started) {
                g1_add_q(acc, acc, sPhi, (nib & 8u) != 0);
            } else {
                sPhi.load(acc);
                if (nib & 8u) f_neg(acc.y, acc.y);
            }
            started = true;
        }
    }
    if (negate) f_neg(acc.y, acc.y);
}

// register-only convenience form (setup-time and element-wise kernels): uses
// a local 72-word scratch as the two slots
template <class ProgPtr>
FK_HD void g1_mul_prog(G1P &R, const G1P &P, ProgPtr prog) {
    uint32_t slots[72];
    StridedPoint sP{slots, 1}, sPhi{slots + 36, 1};
    sP.put(P);
    g1_mul_prog(R, sP, sPhi, prog);
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
        // r = (r << 1) | a_bit
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

// NAF digits of a < 2^128 into d[0..PROG_POSITIONS); returns top position or -1
inline int naf128(int8_t *d, unsigned __int128 k) {
    int top = -1;
    for (int i = 0; i < PROG_POSITIONS; i++) d[i] = 0;
    for (int i = 0; k != 0; i++) {
        if (k & 1) {
            int v = 2 - (int)(k & 3);  // +1 or -1
            d[i] = (int8_t)v;
            if (v > 0) k -= 1; else k += 1;
            top = i;
        }
        k >>= 1;
    }
    return top;
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
    int t1 = naf128(d1, k1), t2 = naf128(d2, k2);
    int top = t1 > t2 ? t1 : t2;
    prog[0] = (uint32_t)top;
    for (int p = 0; p <= top; p++) {
        uint32_t nib = 0;
        if (d1[p]) nib |= 1u | (d1[p] < 0 ? 2u : 0u);
        if (d2[p]) nib |= 4u | (d2[p] < 0 ? 8u : 0u);
        prog[1 + (p >> 3)] |= nib << ((p & 7) * 4);
    }
}

inline void program_cost(const uint32_t prog[PROG_WORDS], int *dbl, int *add);

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
    if (8 * d1 + 12 * a1 < 8 * d0 + 12 * a0) {
        alt[0] |= 0x400u;
        for (int i = 0; i < PROG_WORDS; i++) prog[i] = alt[i];
    }
}

// algorithmic cost of a program in RCB units: doublings and additions
inline void program_cost(const uint32_t prog[PROG_WORDS], int *dbl, int *add) {
    *dbl = *add = 0;
    if (prog[0] & 0x300u) return;
    int top = (int)(prog[0] & 0xff);
    bool started = false;
    for (int p = top; p >= 0; p--) {
        if (started) (*dbl)++;
        uint32_t nib = (prog[1 + (p >> 3)] >> ((p & 7) * 4)) & 0xf;
        if (nib & 1) { if (started) (*add)++; started = true; }
        if (nib & 4) { if (started) (*add)++; started = true; }
    }
}

}  // namespace host

}  // namespace fk
