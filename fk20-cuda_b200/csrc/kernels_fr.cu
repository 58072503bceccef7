// kernels_fr.cu -- Fr side of the pipeline: toeplitz gather fused with the
// 16 Fr FFTs of each row (fk20_poly2toeplitz_coefficients.cu:25-58 followed
// by fr_fft.cu:28-158), plus the reference-layout Fr FFT and toeplitz entry
// points.  Fr data stays in standard form; twiddles are Montgomery constants,
// so Montgomery products of data by twiddles return standard form.
#include "consts.cuh"
#include "glv.cuh"
#include "launch.h"
#include "layout.cuh"

namespace fk {

cudaError_t upload_consts_fr() { return upload_module_consts(); }

// In-place radix-2 DIT over sm[m][8] (bit-reversed input, natural output),
// called by m/2 threads; `inverse` uses w^-t and no 1/m.
__device__ void fr_fft_smem(uint32_t (*sm)[8], int log_m, bool inverse) {
    const int tid = threadIdx.x;
    for (int s = 0; s < log_m; s++) {
        const int half = 1 << s;
        const int j = tid & (half - 1);
        const int i0 = ((tid >> s) << (s + 1)) | j;
        const int i1 = i0 + half;
        Fr u, v, t;
#pragma unroll
        for (int k = 0; k < 8; k++) { u.w[k] = sm[i0][k]; v.w[k] = sm[i1][k]; }
        const int texp = j << (log_m - 1 - s);  // power of w_m
        if (texp != 0) {
            int tix = (texp << (MAX_LOG_M - log_m)) & 511;  // power of w_512
            if (inverse) tix = (512 - tix) & 511;
#pragma unroll
            for (int k = 0; k < 8; k++) t.w[k] = g_fr_tw[tix][k];
            f_mul(v, v, t);
        }
        Fr x, y;
        f_add(x, u, v);
        f_sub(y, u, v);
#pragma unroll
        for (int k = 0; k < 8; k++) { sm[i0][k] = x.w[k]; sm[i1][k] = y.w[k]; }
        __syncthreads();
    }
}

// toeplitz coefficient p of column i for a row of n = 16 k coefficients
// (FK20Py/fk20_multi_cuda.py:145-146; fk20_poly2toeplitz_coefficients.cu:40-56):
//   p = 0: poly[n-1-i];  1 <= p <= k+1: 0;  p = k+2+t: poly[2l-1-i + l t]
__device__ void toeplitz_coef(Fr &v, const uint64_t *__restrict__ poly, int n, int i, int p) {
    const int k = n / L_COLS;
    if (p == 0) {
        fr_from_ref(v, poly + 4 * (size_t)(n - 1 - i));
    } else if (p <= k + 1) {
        f_set_zero(v);
    } else {
        fr_from_ref(v, poly + 4 * (size_t)(2 * L_COLS - 1 - i + L_COLS * (p - k - 2)));
    }
}

// A scalar tile entry holds the GLV halves of the canonical scalar v:
// uint4 0 = v mod lambda, uint4 1 (32 entries on) = v div lambda
// (glv.cuh); the MSM's tables cover 128-bit scalars.
__device__ __forceinline__ void store_scalar(uint4 *dst, const uint32_t v[8]) {
    uint32_t s1[4], s2[4];
    glv_split(s1, s2, v);
    dst[0] = make_uint4(s1[0], s1[1], s1[2], s1[3]);
    dst[32] = make_uint4(s2[0], s2[1], s2[2], s2[3]);
}

// grid (rows, 16), block m/2: toeplitz -> FFT -> scalar tiles S[g][c][i][q][lane]
__global__ void __launch_bounds__(256) k_tc_fft(uint4 *__restrict__ S, const uint64_t *__restrict__ poly,
                                               const size_t *__restrict__ row_off, int n, int log_m) {
    __shared__ uint32_t sm[512][8];
    const int m = 1 << log_m;
    const int row = blockIdx.x, i = blockIdx.y, tid = threadIdx.x;
    const uint64_t *pr = poly + 4 * (row_off ? row_off[row] : (size_t)row * n);
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int p = tid + h * (m >> 1);
        Fr v;
        toeplitz_coef(v, pr, n, i, p);
        const int d = (int)bitrev((unsigned)p, log_m);
#pragma unroll
        for (int k = 0; k < 8; k++) sm[d][k] = v.w[k];
    }
    __syncthreads();
    fr_fft_smem(sm, log_m, false);
    const int g = row >> 5, lane = row & 31;
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int c = tid + h * (m >> 1);
        store_scalar(S + ((((size_t)g * m + c) * L_COLS + i) * SCAL_Q) * 32 + lane, sm[c]);
    }
}

// grid (count), block m/2: batched Fr FFT on reference arrays, natural order in
// and out (fr_fft_wrapper / fr_ift_wrapper, fr_fft.cu:318-363); the inverse
// includes 1/m.  Each block reads its whole transform before writing, so
// in-place calls are safe.
__global__ void __launch_bounds__(256) k_fr_fft_ref(uint64_t *out, const uint64_t *in, int log_m, int inverse) {
    __shared__ uint32_t sm[512][8];
    const int m = 1 << log_m;
    const int tid = threadIdx.x;
    const uint64_t *src = in + 4 * (size_t)blockIdx.x * m;
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int p = tid + h * (m >> 1);
        Fr v;
        fr_from_ref(v, src + 4 * (size_t)p);
        const int d = (int)bitrev((unsigned)p, log_m);
#pragma unroll
        for (int k = 0; k < 8; k++) sm[d][k] = v.w[k];
    }
    __syncthreads();
    fr_fft_smem(sm, log_m, inverse != 0);
    uint64_t *dst = out + 4 * (size_t)blockIdx.x * m;
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int c = tid + h * (m >> 1);
        Fr v;
#pragma unroll
        for (int k = 0; k < 8; k++) v.w[k] = sm[c][k];
        if (inverse) {
            Fr s;
#pragma unroll
            for (int k = 0; k < 8; k++) s.w[k] = g_fr_inv2[log_m][k];
            f_mul(v, v, s);
        }
        fr_to_ref(dst + 4 * (size_t)c, v);
    }
}

// grid (rows), block 256: reference toeplitz output tc[row][16][m], canonical
__global__ void k_toeplitz_ref(uint64_t *__restrict__ tc, const uint64_t *__restrict__ poly, int n, int log_m) {
    const int m = 1 << log_m;
    const int row = blockIdx.x;
    const uint64_t *pr = poly + 4 * (size_t)row * n;
    uint64_t *dst = tc + 4 * (size_t)row * L_COLS * m;
    for (int e = threadIdx.x; e < L_COLS * m; e += blockDim.x) {
        Fr v;
        toeplitz_coef(v, pr, n, e / m, e % m);
        fr_to_ref(dst + 4 * (size_t)e, v);
    }
}

// grid-stride: reference tc_fft[row][16][m] -> scalar tiles (canonicalised)
__global__ void k_ref_to_scalars(uint4 *__restrict__ S, const uint64_t *__restrict__ tcf, int rows, int log_m) {
    const int m = 1 << log_m;
    const size_t total = (size_t)rows * L_COLS * m;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int row = (int)(e / ((size_t)L_COLS * m));
        const int rem = (int)(e % ((size_t)L_COLS * m));
        const int i = rem / m, c = rem % m;
        Fr v;
        fr_from_ref(v, tcf + 4 * e);
        const int g = row >> 5, lane = row & 31;
        store_scalar(S + ((((size_t)g * m + c) * L_COLS + i) * SCAL_Q) * 32 + lane, v.w);
    }
}

void launch_tc_fft(uint4 *S, const uint64_t *poly, const size_t *row_off, int n, int log_m, unsigned rows,
                   cudaStream_t st) {
    k_tc_fft<<<dim3(rows, L_COLS), (1u << log_m) / 2, 0, st>>>(S, poly, row_off, n, log_m);
}
void launch_fr_fft_ref(uint64_t *out, const uint64_t *in, int log_m, unsigned count, int inverse, cudaStream_t st) {
    k_fr_fft_ref<<<count, (1u << log_m) / 2, 0, st>>>(out, in, log_m, inverse);
}
void launch_toeplitz_ref(uint64_t *tc, const uint64_t *poly, int n, int log_m, unsigned rows, cudaStream_t st) {
    k_toeplitz_ref<<<rows, 256, 0, st>>>(tc, poly, n, log_m);
}
void launch_ref_to_scalars(uint4 *S, const uint64_t *tcf, int rows, int log_m, cudaStream_t st) {
    k_ref_to_scalars<<<grid_stride_blocks((size_t)rows * L_COLS * (1u << log_m)), 256, 0, st>>>(S, tcf, rows, log_m);
}

}  // namespace fk
