// kernels_out.cu -- proofs in the data-availability wire format.
//
// A proof leaves the engine as the 48-byte compressed encoding of its affine
// point (the BLS12-381 serialization of the ZCash/IETF convention): x as 48
// big-endian bytes, whose top three bits are flags -- 0x80 compressed, 0x40
// point at infinity (all other bits zero), 0x20 y is the larger of y and p - y.
// In data-availability order the proofs of a row are bit-reversed
// (FK20Py/fk20_multi_cuda.py:249-260, list_to_reverse_bit_order in
// FK20Py/kzg_proofs.py:105-118): output i of a row is h_fft[bitrev(i)].
#include "launch.h"
#include "layout.cuh"

namespace fk {

// bswap of a 32-bit word (big-endian byte order in memory)
FK_D uint32_t be32(uint32_t v) { return __byte_perm(v, 0, 0x0123); }

// 48-byte encoding of p as 12 words in memory order
FK_D void g1_compress48(uint32_t out[12], const G1P &p) {
    if (f_is_zero(p.z)) {
        out[0] = 0xc0u;  // bytes c0 00 00 00
#pragma unroll
        for (int k = 1; k < 12; k++) out[k] = 0;
        return;
    }
    G1P a = p;
    g1_normalize(a);  // z = 1 (Montgomery): one inversion
    Fp x, y;
    f_from_mont(x, a.x);
    f_from_mont(y, a.y);
    // y > (p - 1) / 2  <=>  2y >= p  (2y < 2^383, no overflow of 12 words + carry)
    uint32_t t[12], s[12];
    ch_add<FpDesc>(t, y.w, y.w);
    const uint32_t borrow = ch_sub_mod<FpDesc>(s, t);  // all ones when 2y < p
#pragma unroll
    for (int k = 0; k < 12; k++) out[k] = be32(x.w[11 - k]);
    out[0] |= 0x80u | (borrow ? 0u : 0x20u);
}

FK_D void store48(uint8_t *dst, const uint32_t w[12]) {
    uint4 *d = reinterpret_cast<uint4 *>(dst);
    d[0] = make_uint4(w[0], w[1], w[2], w[3]);
    d[1] = make_uint4(w[4], w[5], w[6], w[7]);
    d[2] = make_uint4(w[8], w[9], w[10], w[11]);
}

__global__ void k_g1p_compress(uint8_t *__restrict__ out, const uint64_t *__restrict__ pin, size_t count) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < count; e += (size_t)gridDim.x * blockDim.x) {
        G1P p;
        g1p_from_ref(p, pin + 18 * e);
        uint32_t w[12];
        g1_compress48(w, p);
        store48(out + 48 * e, w);
    }
}

// h_fft[rows][m] (reference layout) -> proofs[rows][m][48] in data-availability order
__global__ void k_h_fft_to_proofs(uint8_t *__restrict__ out, const uint64_t *__restrict__ h, int rows, int log_m) {
    const int m = 1 << log_m;
    const size_t total = (size_t)rows * m;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const size_t row = e >> log_m;
        const int i = (int)(e & (m - 1));
        G1P p;
        g1p_from_ref(p, h + 18 * ((row << log_m) + bitrev((unsigned)i, log_m)));
        uint32_t w[12];
        g1_compress48(w, p);
        store48(out + 48 * e, w);
    }
}

// pipeline tiles (h_fft, natural order) -> proofs in data-availability order;
// row r's proofs start at proof index (out_off ? out_off[r] : r * m)
__global__ void k_tile_to_proofs(uint8_t *__restrict__ out, const uint4 *__restrict__ D,
                                 const size_t *__restrict__ out_off, int rows, int log_m) {
    const int m = 1 << log_m;
    const size_t total = (size_t)rows * m;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int row = (int)(e >> log_m), i = (int)(e & (m - 1));
        G1P p;
        tile_load(p, D + tile_index(row >> 5, m, (int)bitrev((unsigned)i, log_m)), row & 31);
        uint32_t w[12];
        g1_compress48(w, p);
        const size_t base = out_off ? out_off[row] : (size_t)row * m;
        store48(out + 48 * (base + i), w);
    }
}

void launch_g1p_compress(uint8_t *out, const uint64_t *p, size_t count, cudaStream_t st) {
    k_g1p_compress<<<grid_stride_blocks(count), 128, 0, st>>>(out, p, count);
}
void launch_h_fft_to_proofs(uint8_t *out, const uint64_t *h, int rows, int log_m, cudaStream_t st) {
    k_h_fft_to_proofs<<<grid_stride_blocks((size_t)rows << log_m), 128, 0, st>>>(out, h, rows, log_m);
}
void launch_tile_to_proofs(uint8_t *out, const uint4 *D, const size_t *out_off, int rows, int log_m,
                           cudaStream_t st) {
    k_tile_to_proofs<<<grid_stride_blocks((size_t)rows << log_m), 128, 0, st>>>(out, D, out_off, rows, log_m);
}

}  // namespace fk
