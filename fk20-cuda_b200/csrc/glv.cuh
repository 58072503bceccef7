// glv.cuh -- the GLV split of an Fr scalar for the fixed-base MSM.
//
// phi(x, y) = (beta x, y) acts on G1 as [lambda] with lambda = z^2 - 1
// (z = -0xd201000000010000, the BLS12-381 parameter) and
// lambda^2 + lambda + 1 = r.  Any s < r is s1 + s2 lambda with
// s1 = s mod lambda and s2 = s div lambda, both below 2^128, so
// [s] X = [s1] X + [s2] phi(X): the fixed-base tables only have to cover
// 128-bit scalars (half the windows), and phi costs one product.
#pragma once
#include "field.cuh"

namespace fk {

// lambda = GLV_LAMBDA1 2^64 + GLV_LAMBDA0
constexpr uint64_t GLV_LAMBDA0 = 0x00000000ffffffffull, GLV_LAMBDA1 = 0xac45a4010001a402ull;
// floor(2^256 / lambda) = 2^128 + GLV_MU1 2^64 + GLV_MU0
constexpr uint64_t GLV_MU0 = 0x63f6e522f6cfee30ull, GLV_MU1 = 0x7c6becf1e01faaddull;

FK_HD uint64_t glv_mulhi(uint64_t a, uint64_t b) {
#if defined(__CUDA_ARCH__)
    return __umul64hi(a, b);
#else
    return (uint64_t)(((unsigned __int128)a * b) >> 64);
#endif
}

// s = s1 + s2 lambda with s1 = s mod lambda, s2 = s div lambda, for
// s < 2^255 given as 8 little-endian 32-bit words; s1 and s2 are 4 words
// each.  Barrett division: with t = s >> 126 and mu = floor(2^256 / lambda),
// q = (t mu) >> 130 is s div lambda or at most 2 below it
// (t > s / 2^126 - 1, mu > 2^256 / lambda - 1, s < 2^255, lambda > 2^127),
// and two conditional subtractions of lambda finish it.
FK_HD void glv_split(uint32_t s1[4], uint32_t s2[4], const uint32_t s[8]) {
    uint64_t a[4];
#pragma unroll
    for (int k = 0; k < 4; k++) a[k] = (uint64_t)s[2 * k] | ((uint64_t)s[2 * k + 1] << 32);
    const uint64_t t[3] = {(a[1] >> 62) | (a[2] << 2), (a[2] >> 62) | (a[3] << 2), a[3] >> 62};
    const uint64_t mu[3] = {GLV_MU0, GLV_MU1, 1};
    uint64_t p[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int i = 0; i < 3; i++) {
        uint64_t carry = 0;
#pragma unroll
        for (int j = 0; j < 3; j++) {
            // p[i + j] + t[i] mu[j] + carry < 2^128: the new carry fits a word
            const uint64_t lo = t[i] * mu[j], hi = glv_mulhi(t[i], mu[j]);
            uint64_t x = p[i + j] + lo;
            uint64_t c = x < lo;
            x += carry;
            c += x < carry;
            p[i + j] = x;
            carry = hi + c;
        }
        p[i + 3] = carry;
    }
    uint64_t q0 = (p[2] >> 2) | (p[3] << 62), q1 = (p[3] >> 2) | (p[4] << 62);
    // r = s - q lambda (r < 3 lambda < 2^130: three words)
    const uint64_t l[2] = {GLV_LAMBDA0, GLV_LAMBDA1};
    const uint64_t q[2] = {q0, q1};
    uint64_t ql[4] = {0, 0, 0, 0};
#pragma unroll
    for (int i = 0; i < 2; i++) {
        uint64_t carry = 0;
#pragma unroll
        for (int j = 0; j < 2; j++) {
            const uint64_t lo = q[i] * l[j], hi = glv_mulhi(q[i], l[j]);
            uint64_t x = ql[i + j] + lo;
            uint64_t c = x < lo;
            x += carry;
            c += x < carry;
            ql[i + j] = x;
            carry = hi + c;
        }
        ql[i + 2] = carry;
    }
    uint64_t r[3];
    uint64_t br = 0;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const uint64_t d = a[k] - ql[k];
        const uint64_t b1 = a[k] < ql[k];
        r[k] = d - br;
        br = b1 | (d < br);
    }
#pragma unroll
    for (int it = 0; it < 2; it++) {
        const bool ge = r[2] != 0 || r[1] > l[1] || (r[1] == l[1] && r[0] >= l[0]);
        if (ge) {
            const uint64_t d0 = r[0] - l[0], b0 = r[0] < l[0];
            const uint64_t d1 = r[1] - l[1], b1 = r[1] < l[1];
            r[0] = d0;
            r[1] = d1 - b0;
            r[2] -= b1 | (d1 < b0);
            q0 += 1;
            q1 += q0 == 0;
        }
    }
    s1[0] = (uint32_t)r[0];
    s1[1] = (uint32_t)(r[0] >> 32);
    s1[2] = (uint32_t)r[1];
    s1[3] = (uint32_t)(r[1] >> 32);
    s2[0] = (uint32_t)q0;
    s2[1] = (uint32_t)(q0 >> 32);
    s2[2] = (uint32_t)q1;
    s2[3] = (uint32_t)(q1 >> 32);
}

}  // namespace fk
