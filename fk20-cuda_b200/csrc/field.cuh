// field.cuh -- BLS12-381 Fp (381-bit) and Fr (255-bit) Montgomery arithmetic.
//
// Elements are little-endian arrays of 32-bit limbs (Fp: 12, Fr: 8).  Inside
// the engine Fp values are in Montgomery form (x*2^384 mod p) and always
// canonical (< p); Fr data keeps its standard form and is multiplied by
// Montgomery-form constants (x*y*2^-256 with y = w*2^256 gives x*w), so Fr
// FFT outputs are standard-form without conversions.  The reference stores
// plain (non-Montgomery) values with Barrett reduction (fp.cuh:10-14,
// fr.cuh:10-24, fr_mul.cu:58-186); conversion happens at the ABI boundary.
//
// Montgomery product r = A*B/2^(32N): word-serial CIOS with the partial products of each
// word b_i split between two accumulators, `e` (products a_j*b_i with j even:
// lo at word j, hi at word j+1) and `o` (j odd).  Within one accumulator the
// lo/hi words of different j never overlap, so each half is a single
// mad.lo.cc/madc.hi.cc carry chain and the two chains are independent.  The
// reduction multiple m*p is split the same way.  After the reduction the
// word-0 sum e0+o0 is 0 mod 2^32; its carry (0 or 1) is fed into the next
// iteration at word 0 of the odd chain, and both accumulators shift down one
// word.  Bounds: with A < 2p (4p < 2^384) and B < 2^384 every partial value
// stays below 2^416, so 13 words per accumulator suffice, and the result is
// < 2p when A, B < 2p or when A < p (one conditional subtraction of p makes
// it canonical).  A must not exceed ~2^382: a full-width A overflows.
#pragma once
#include "limbs.cuh"

namespace fk {

// ---------------------------------------------------------------- moduli
struct FpDesc {
    static constexpr int N = 12;
    static constexpr uint32_t M0 = 0xfffcfffdu;  // -p^-1 mod 2^32
    FK_HD static constexpr uint32_t mod(int i) {
        return i == 0 ? 0xffffaaabu : i == 1 ? 0xb9feffffu : i == 2 ? 0xb153ffffu : i == 3 ? 0x1eabfffeu
             : i == 4 ? 0xf6b0f624u : i == 5 ? 0x6730d2a0u : i == 6 ? 0xf38512bfu : i == 7 ? 0x64774b84u
             : i == 8 ? 0x434bacd7u : i == 9 ? 0x4b1ba7b6u : i == 10 ? 0x397fe69au : 0x1a0111eau;
    }
    // 2^768 mod p (to Montgomery form)
    FK_HD static constexpr uint32_t r2(int i) {
        return i == 0 ? 0x1c341746u : i == 1 ? 0xf4df1f34u : i == 2 ? 0x09d104f1u : i == 3 ? 0x0a76e6a6u
             : i == 4 ? 0x4c95b6d5u : i == 5 ? 0x8de5476cu : i == 6 ? 0x939d83c0u : i == 7 ? 0x67eb88a9u
             : i == 8 ? 0xb519952du : i == 9 ? 0x9a793e85u : i == 10 ? 0x92cae3aau : 0x11988fe5u;
    }
    // 2^384 mod p (Montgomery one)
    FK_HD static constexpr uint32_t one(int i) {
        return i == 0 ? 0x0002fffdu : i == 1 ? 0x76090000u : i == 2 ? 0xc40c0002u : i == 3 ? 0xebf4000bu
             : i == 4 ? 0x53c758bau : i == 5 ? 0x5f489857u : i == 6 ? 0x70525745u : i == 7 ? 0x77ce5853u
             : i == 8 ? 0xa256ec6du : i == 9 ? 0x5c071a97u : i == 10 ? 0xfa80e493u : 0x15f65ec3u;
    }
};

struct FrDesc {
    static constexpr int N = 8;
    static constexpr uint32_t M0 = 0xffffffffu;  // -r^-1 mod 2^32
    FK_HD static constexpr uint32_t mod(int i) {
        return i == 0 ? 0x00000001u : i == 1 ? 0xffffffffu : i == 2 ? 0xfffe5bfeu : i == 3 ? 0x53bda402u
             : i == 4 ? 0x09a1d805u : i == 5 ? 0x3339d808u : i == 6 ? 0x299d7d48u : 0x73eda753u;
    }
    FK_HD static constexpr uint32_t r2(int i) {
        return i == 0 ? 0xf3f29c6du : i == 1 ? 0xc999e990u : i == 2 ? 0x87925c23u : i == 3 ? 0x2b6cedcbu
             : i == 4 ? 0x7254398fu : i == 5 ? 0x05d31496u : i == 6 ? 0x9f59ff11u : 0x0748d9d9u;
    }
    FK_HD static constexpr uint32_t one(int i) {
        return i == 0 ? 0xfffffffeu : i == 1 ? 0x00000001u : i == 2 ? 0x00034802u : i == 3 ? 0x5884b7fau
             : i == 4 ? 0xecbc4ff5u : i == 5 ? 0x998c4fefu : i == 6 ? 0xacc5056fu : 0x1824b159u;
    }
};

template <class F>
struct Elem {
    uint32_t w[F::N];
};
using Fp = Elem<FpDesc>;
using Fr = Elem<FrDesc>;

// ---------------------------------------------------------------- carry chains
// Each chain is one inline-PTX statement in device code (chains.inc, written
// by gen_chains.py): the carry flag CC.CF never has to survive from one asm
// statement to the next.  Host builds run the portable stand-ins below, which
// compute the same words.
template <class F> FK_D void ptx_add(uint32_t *r, const uint32_t *a, const uint32_t *b);
template <class F> FK_D uint32_t ptx_sub(uint32_t *r, const uint32_t *a, const uint32_t *b);
template <class F> FK_D uint32_t ptx_sub_mod(uint32_t *r, const uint32_t *t);
template <class F> FK_D void ptx_row_even(uint32_t *e, const uint32_t *a, uint32_t b);
template <class F> FK_D void ptx_row_odd(uint32_t *o, const uint32_t *a, uint32_t b, uint32_t c);
template <class F> FK_D void ptx_red_even(uint32_t *e, uint32_t m);
template <class F> FK_D void ptx_red_odd(uint32_t *o, uint32_t m);
template <class F> FK_D void ptx_final(uint32_t *t, const uint32_t *e, const uint32_t *o);
template <class F> FK_D void ptx_final_c(uint32_t *t, const uint32_t *e, const uint32_t *o, uint32_t c);
template <class F, int I> FK_D void ptx_sqrow_even(uint32_t *e, const uint32_t *v, uint32_t b);
template <class F, int I> FK_D void ptx_sqrow_odd(uint32_t *o, const uint32_t *v, uint32_t b);
#if defined(__CUDA_ARCH__)
#include "chains.inc"
#endif

// r = a + b; the carry out of the top word is dropped (callers keep sums < 2^(32N))
template <class F>
FK_HD void ch_add(uint32_t *r, const uint32_t *a, const uint32_t *b) {
#if defined(__CUDA_ARCH__)
    ptx_add<F>(r, a, b);
#else
    uint64_t c = 0;
    for (int i = 0; i < F::N; i++) { c += (uint64_t)a[i] + b[i]; r[i] = (uint32_t)c; c >>= 32; }
#endif
}

// r = a - b; returns all ones when a < b, else 0
template <class F>
FK_HD uint32_t ch_sub(uint32_t *r, const uint32_t *a, const uint32_t *b) {
#if defined(__CUDA_ARCH__)
    return ptx_sub<F>(r, a, b);
#else
    uint64_t br = 0;
    for (int i = 0; i < F::N; i++) { uint64_t d = (uint64_t)a[i] - b[i] - br; r[i] = (uint32_t)d; br = d >> 63; }
    return br ? 0xffffffffu : 0u;
#endif
}

// r = t - modulus; returns all ones when t < modulus, else 0
template <class F>
FK_HD uint32_t ch_sub_mod(uint32_t *r, const uint32_t *t) {
#if defined(__CUDA_ARCH__)
    return ptx_sub_mod<F>(r, t);
#else
    uint32_t m[F::N];
    for (int i = 0; i < F::N; i++) m[i] = F::mod(i);
    return ch_sub<F>(r, t, m);
#endif
}

// e[0..N-1] += a[j]*b for even j (lo word at j, hi word at j+1); e[N] = carry out
template <class F>
FK_HD void ch_row_even(uint32_t *e, const uint32_t *a, uint32_t b) {
#if defined(__CUDA_ARCH__)
    ptx_row_even<F>(e, a, b);
#else
    uint64_t c = 0;
    for (int w = 0; w < F::N; w++) {
        c += (uint64_t)e[w] + ((w & 1) ? mul_hi(a[w - 1], b) : mul_lo(a[w], b));
        e[w] = (uint32_t)c;
        c >>= 32;
    }
    e[F::N] = (uint32_t)c;
#endif
}

// o[0] += c; o[1..N] += a[j]*b for odd j (lo word at j, hi word at j+1);
// o[N] is written, not read
template <class F>
FK_HD void ch_row_odd(uint32_t *o, const uint32_t *a, uint32_t b, uint32_t c) {
#if defined(__CUDA_ARCH__)
    ptx_row_odd<F>(o, a, b, c);
#else
    uint64_t s = (uint64_t)o[0] + c;
    o[0] = (uint32_t)s;
    s >>= 32;
    for (int w = 1; w < F::N; w++) {
        s += (uint64_t)o[w] + ((w & 1) ? mul_lo(a[w], b) : mul_hi(a[w - 1], b));
        o[w] = (uint32_t)s;
        s >>= 32;
    }
    o[F::N] = (uint32_t)(s + mul_hi(a[F::N - 1], b));
#endif
}

// e[0..N-1] += m*mod[j] for even j; e[N] += carry out
template <class F>
FK_HD void ch_red_even(uint32_t *e, uint32_t m) {
#if defined(__CUDA_ARCH__)
    ptx_red_even<F>(e, m);
#else
    uint64_t c = 0;
    for (int w = 0; w < F::N; w++) {
        c += (uint64_t)e[w] + ((w & 1) ? mul_hi(m, F::mod(w - 1)) : mul_lo(m, F::mod(w)));
        e[w] = (uint32_t)c;
        c >>= 32;
    }
    e[F::N] += (uint32_t)c;
#endif
}

// o[1..N] += m*mod[j] for odd j (o[0] unchanged)
template <class F>
FK_HD void ch_red_odd(uint32_t *o, uint32_t m) {
#if defined(__CUDA_ARCH__)
    ptx_red_odd<F>(o, m);
#else
    uint64_t c = 0;
    for (int w = 1; w < F::N; w++) {
        c += (uint64_t)o[w] + ((w & 1) ? mul_lo(m, F::mod(w)) : mul_hi(m, F::mod(w - 1)));
        o[w] = (uint32_t)c;
        c >>= 32;
    }
    o[F::N] += (uint32_t)c + mul_hi(m, F::mod(F::N - 1));
#endif
}

// t[0..N-1] = (e + o) >> 32 over N+1 words
template <class F>
FK_HD void ch_final(uint32_t *t, const uint32_t *e, const uint32_t *o) {
#if defined(__CUDA_ARCH__)
    ptx_final<F>(t, e, o);
#else
    uint64_t c = ((uint64_t)e[0] + o[0]) >> 32;
    for (int k = 1; k <= F::N; k++) {
        c += (uint64_t)e[k] + o[k];
        t[k - 1] = (uint32_t)c;
        c >>= 32;
    }
#endif
}

// t[0..N-1] = (e + o + c) >> 32 over N+1 words, c (0 or 1) added at word 0
template <class F>
FK_HD void ch_final_c(uint32_t *t, const uint32_t *e, const uint32_t *o, uint32_t c) {
#if defined(__CUDA_ARCH__)
    ptx_final_c<F>(t, e, o, c);
#else
    uint64_t s = ((uint64_t)e[0] + o[0] + c) >> 32;
    for (int k = 1; k <= F::N; k++) {
        s += (uint64_t)e[k] + o[k];
        t[k - 1] = (uint32_t)s;
        s >>= 32;
    }
#endif
}

// squaring row I >= 1, one parity P of j (0: the e half, 1: the o half):
// acc[j0..] += v[j] * b for j >= I, j = P mod 2 (lo word at j, hi word at
// j + 1), the carry out of the e half into e[N]; acc[N] is written, not read
template <class F, int I, int P>
FK_HD void ch_sqrow(uint32_t *acc, const uint32_t *v, uint32_t b) {
#if defined(__CUDA_ARCH__)
    if (P == 0) ptx_sqrow_even<F, I>(acc, v, b);
    else ptx_sqrow_odd<F, I>(acc, v, b);
#else
    constexpr int N = F::N;
    const int j0 = (I % 2 == P) ? I : I + 1;
    if (j0 >= N) return;  // no product of this parity (acc[N] keeps its 0)
    uint64_t c = 0;
    for (int w = j0; w < N; w++) {
        c += (uint64_t)acc[w] + (((w - j0) & 1) ? mul_hi(v[w - 1], b) : mul_lo(v[w], b));
        acc[w] = (uint32_t)c;
        c >>= 32;
    }
    acc[N] = P == 0 ? (uint32_t)c : (uint32_t)(c + mul_hi(v[N - 1], b));
#endif
}

// the carry out of e0 + o0 + c, c = 0 or 1
FK_HD uint32_t ch_carry3(uint32_t e0, uint32_t o0, uint32_t c) {
#if defined(__CUDA_ARCH__)
    return ptx_carry3(e0, o0, c);
#else
    return (uint32_t)(((uint64_t)e0 + o0 + c) >> 32);
#endif
}

// the carry out of e0 + o0
FK_HD uint32_t ch_carry0(uint32_t e0, uint32_t o0) {
#if defined(__CUDA_ARCH__)
    return ptx_carry0(e0, o0);
#else
    return (uint32_t)(((uint64_t)e0 + o0) >> 32);
#endif
}

// ---------------------------------------------------------------- helpers
template <class F>
FK_HD void f_set_zero(Elem<F> &r) {
#pragma unroll
    for (int i = 0; i < F::N; i++) r.w[i] = 0;
}

template <class F>
FK_HD void f_set_one(Elem<F> &r) {  // Montgomery one
#pragma unroll
    for (int i = 0; i < F::N; i++) r.w[i] = F::one(i);
}

template <class F>
FK_HD bool f_is_zero(const Elem<F> &a) {
    uint32_t o = 0;
#pragma unroll
    for (int i = 0; i < F::N; i++) o |= a.w[i];
    return o == 0;
}

template <class F>
FK_HD bool f_eq(const Elem<F> &a, const Elem<F> &b) {
    uint32_t o = 0;
#pragma unroll
    for (int i = 0; i < F::N; i++) o |= a.w[i] ^ b.w[i];
    return o == 0;
}

// r = t - mod if t >= mod else t   (t < 2*mod < 2^(32N))
template <class F>
FK_HD void f_reduce_once(uint32_t r[F::N], const uint32_t t[F::N]) {
    constexpr int N = F::N;
    uint32_t s[N];
    const uint32_t borrow = ch_sub_mod<F>(s, t);  // 0xffffffff if t < mod
#pragma unroll
    for (int i = 0; i < N; i++) r[i] = (t[i] & borrow) | (s[i] & ~borrow);
}

// ---------------------------------------------------------------- Montgomery product
template <class F>
FK_HD void f_mul(Elem<F> &r, const Elem<F> &A, const Elem<F> &B) {
    constexpr int N = F::N;
    const uint32_t *a = A.w;
    uint32_t e[N + 1], o[N + 1];
    uint32_t c = 0;

    // word 0 of b: plain products, no chains needed
    {
        const uint32_t bi = B.w[0];
#pragma unroll
        for (int j = 0; j < N; j += 2) {
            e[j] = mul_lo(a[j], bi);
            e[j + 1] = mul_hi(a[j], bi);
        }
        e[N] = 0;
        o[0] = 0;
#pragma unroll
        for (int j = 1; j < N; j += 2) {
            o[j] = mul_lo(a[j], bi);
            o[j + 1] = mul_hi(a[j], bi);
        }
    }

#pragma unroll
    for (int i = 0; i < N; i++) {
        if (i > 0) {
            // even products into e[0..N]; the previous word-0 carry and the
            // odd products into o[0..N]
            ch_row_even<F>(e, a, B.w[i]);
            ch_row_odd<F>(o, a, B.w[i], c);
        }
        // reduction: add m*p, m chosen so that word 0 vanishes
        const uint32_t m = mul_lo(e[0] + o[0], F::M0);
        ch_red_even<F>(e, m);
        ch_red_odd<F>(o, m);
        if (i < N - 1) {
            c = ch_carry0(e[0], o[0]);
#pragma unroll
            for (int k = 0; k < N; k++) {
                e[k] = e[k + 1];
                o[k] = o[k + 1];
            }
            e[N] = 0;
            o[N] = 0;
        }
    }
    // final: (e + o) >> 32, then one conditional subtraction
    uint32_t t[N];
    ch_final<F>(t, e, o);
    f_reduce_once<F>(r.w, t);
}

// ---------------------------------------------------------------- Montgomery square
// The same word-serial CIOS as f_mul, with the products of word i of A
// restricted to words j >= i (78 of 144 limb products for Fp, 36 of 64 for
// Fr): row i adds a_i * V_i, V_i = a_i 2^(32 i) + 2 sum_{j > i} a_j 2^(32 j),
// whose words are a_i, a_{i+1} << 1 and then the words of 2A (the top bit of
// a_i belongs to row i's own a_i, not to 2A's word i + 1).  Sum over i:
// sum a_i^2 2^(64 i) + 2 sum_{i<j} a_i a_j 2^(32(i+j)) = A^2.  As a row no
// longer starts at word 0, the word-0 carry c of each reduction step is
// carried into the next step's word-0 sum (and the final shift) instead of
// the odd half's first word.  Bounds: V_i <= 2A, so A < 2^(32N - 2) keeps
// every partial value where f_mul's do (A canonical: A < m), except the top
// word of the odd half, which holds hi(2 a_{N-1} a_i) + hi(m mod_{N-1}) and
// stays below 2^32 only for a modulus whose top word is below 2^30 (Fp:
// 0x1a0111ea; Fr's 0x73eda753 is not, so Fr squares are products).
template <class F, int I>
FK_HD void f_sqr_rows(uint32_t *e, uint32_t *o, uint32_t &c, const uint32_t *a, const uint32_t *a2) {
    constexpr int N = F::N;
    if constexpr (I > 0) {
        uint32_t v[N];
#pragma unroll
        for (int j = 0; j < N; j++) v[j] = j == I ? a[I] : j == I + 1 ? a[I + 1] << 1 : a2[j];
        ch_sqrow<F, I, 0>(e, v, a[I]);
        ch_sqrow<F, I, 1>(o, v, a[I]);
    }
    // reduction: add m*p, m chosen so that word 0 (with the pending carry) vanishes
    const uint32_t m = mul_lo(e[0] + o[0] + c, F::M0);
    ch_red_even<F>(e, m);
    ch_red_odd<F>(o, m);
    if constexpr (I < N - 1) {
        c = ch_carry3(e[0], o[0], c);
#pragma unroll
        for (int k = 0; k < N; k++) {
            e[k] = e[k + 1];
            o[k] = o[k + 1];
        }
        e[N] = 0;
        o[N] = 0;
        f_sqr_rows<F, I + 1>(e, o, c, a, a2);
    }
}

template <class F>
FK_HD void f_sqr(Elem<F> &r, const Elem<F> &A) {
    constexpr int N = F::N;
    if constexpr (F::mod(N - 1) >= (1u << 30)) {
        f_mul<F>(r, A, A);
    } else {
        const uint32_t *a = A.w;
        uint32_t a2[N];  // the words of 2A
        a2[0] = a[0] << 1;
#pragma unroll
        for (int j = 1; j < N; j++) a2[j] = (a[j] << 1) | (a[j - 1] >> 31);
        uint32_t e[N + 1], o[N + 1];
        uint32_t c = 0;
        {
            // row 0: V_0 = (a_0, a_1 << 1, 2A's words 2..N-1), plain products
            const uint32_t b = a[0];
#pragma unroll
            for (int j = 0; j < N; j += 2) {
                const uint32_t v = j == 0 ? a[0] : a2[j];
                e[j] = mul_lo(v, b);
                e[j + 1] = mul_hi(v, b);
            }
            e[N] = 0;
            o[0] = 0;
#pragma unroll
            for (int j = 1; j < N; j += 2) {
                const uint32_t v = j == 1 ? a[1] << 1 : a2[j];
                o[j] = mul_lo(v, b);
                o[j + 1] = mul_hi(v, b);
            }
        }
        f_sqr_rows<F, 0>(e, o, c, a, a2);
        uint32_t t[N];
        ch_final_c<F>(t, e, o, c);
        f_reduce_once<F>(r.w, t);
    }
}

template <class F>
FK_HD void f_add(Elem<F> &r, const Elem<F> &a, const Elem<F> &b) {
    uint32_t t[F::N];
    ch_add<F>(t, a.w, b.w);
    f_reduce_once<F>(r.w, t);
}

template <class F>
FK_HD void f_sub(Elem<F> &r, const Elem<F> &a, const Elem<F> &b) {
    constexpr int N = F::N;
    uint32_t t[N], m[N];
    const uint32_t borrow = ch_sub<F>(t, a.w, b.w);
#pragma unroll
    for (int i = 0; i < N; i++) m[i] = F::mod(i) & borrow;
    ch_add<F>(r.w, t, m);
}

template <class F>
FK_HD void f_neg(Elem<F> &r, const Elem<F> &a) {
    Elem<F> z;
    f_set_zero(z);
    f_sub<F>(r, z, a);
}

template <class F>
FK_HD void f_dbl(Elem<F> &r, const Elem<F> &a) { f_add<F>(r, a, a); }

// r = 12 a  (3b for b = 4)
template <class F>
FK_HD void f_mul12(Elem<F> &r, const Elem<F> &a) {
    Elem<F> t;
    f_add<F>(t, a, a);
    f_add<F>(t, t, a);
    f_add<F>(t, t, t);
    f_add<F>(r, t, t);
}

template <class F>
FK_HD void f_cmov(Elem<F> &r, const Elem<F> &a, bool cond) {
    const uint32_t m = cond ? 0xffffffffu : 0u;
#pragma unroll
    for (int i = 0; i < F::N; i++) r.w[i] = (a.w[i] & m) | (r.w[i] & ~m);
}

// standard form (any value < 2^(32N)) -> Montgomery form, canonical.  The
// reduced constant R^2 mod m goes in the first (multiplicand) slot: f_mul's
// accumulator bound needs that operand below ~2^(32N - 2), while the second
// operand, scanned word by word, may be any 32N-bit value.
template <class F>
FK_HD void f_to_mont(Elem<F> &r, const Elem<F> &a) {
    Elem<F> r2;
#pragma unroll
    for (int i = 0; i < F::N; i++) r2.w[i] = F::r2(i);
    f_mul<F>(r, r2, a);
}

// Montgomery form -> canonical standard form
template <class F>
FK_HD void f_from_mont(Elem<F> &r, const Elem<F> &a) {
    Elem<F> one;
    f_set_zero(one);
    one.w[0] = 1;
    f_mul<F>(r, a, one);
}

// canonical reduction of any standard-form value < 2^(32N)
template <class F>
FK_HD void f_canon(Elem<F> &r, const Elem<F> &a) {
    Elem<F> t;
    f_to_mont<F>(t, a);
    f_from_mont<F>(r, t);
}

// r = a^e for a little-endian exponent of `nw` 32-bit words (Montgomery domain)
template <class F>
FK_HD void f_pow(Elem<F> &r, const Elem<F> &a, const uint32_t *e, int nw) {
    Elem<F> acc;
    f_set_one(acc);
    for (int i = 32 * nw - 1; i >= 0; i--) {
        f_sqr<F>(acc, acc);
        if ((e[i >> 5] >> (i & 31)) & 1) f_mul<F>(acc, acc, a);
    }
    r = acc;
}

// inverse by Fermat's little theorem, a^(m-2); inv(0) = 0
template <class F>
FK_HD void f_inv(Elem<F> &r, const Elem<F> &a) {
    uint32_t e[F::N];
    uint64_t br = 2;
#pragma unroll
    for (int i = 0; i < F::N; i++) {
        const uint64_t d = (uint64_t)F::mod(i) - br;
        e[i] = (uint32_t)d;
        br = d >> 63;
    }
    f_pow<F>(r, a, e, F::N);
}

}  // namespace fk
