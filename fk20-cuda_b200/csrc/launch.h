// launch.h -- host launchers exported by the kernel translation units.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace fk {

struct MsmArgs {
    uint4 *D;
    const uint4 *S;
    const uint4 *table;
    int G, log_m, rows, cb, W, times_m;
};

// per-module constant upload (one per translation unit)
cudaError_t upload_consts_fr();
cudaError_t upload_consts_msm();
cudaError_t upload_consts_fft();
cudaError_t upload_consts_tables();
cudaError_t upload_consts_misc();

// kernels_fr.cu
void launch_tc_fft(uint4 *S, const uint64_t *poly, const size_t *row_off, int n, int log_m, unsigned rows,
                   cudaStream_t st);
void launch_fr_fft_ref(uint64_t *out, const uint64_t *in, int log_m, unsigned count, int inverse, cudaStream_t st);
void launch_toeplitz_ref(uint64_t *tc, const uint64_t *poly, int n, int log_m, unsigned rows, cudaStream_t st);
void launch_ref_to_scalars(uint4 *S, const uint64_t *tcf, int rows, int log_m, cudaStream_t st);

// kernels_msm.cu
void launch_msm(const MsmArgs &a, cudaStream_t st);

// kernels_fft.cu
void launch_g1_stage(uint4 *D, int G, int log_m, int s, int kind, cudaStream_t st);
void launch_g1_middle(uint4 *D, int G, int log_m, int scale, cudaStream_t st);
void launch_g1_fused(uint4 *D, unsigned *ready, unsigned *next, int *err, unsigned epoch, int G, int log_m,
                     int sms, cudaStream_t st);
void launch_g1_scale(uint4 *D, int G, int log_m, int prog, cudaStream_t st);
void launch_ref_to_tile(uint4 *D, const uint64_t *src, int rows, int G, int log_m, int bitrev_in, int zero_upper,
                        cudaStream_t st);
void launch_tile_to_ref(uint64_t *dst, const uint4 *D, const size_t *row_off, int rows, int log_m, int bitrev_out,
                        cudaStream_t st);
void launch_hext2h_ref(uint64_t *h, int rows, int log_m, cudaStream_t st);
void launch_setup_to_tile(uint4 *D, const uint64_t *setup, int n, int log_m, cudaStream_t st);

// kernels_tables.cu
size_t table_window_base_bytes();  // sizeof(G1P)
size_t table_z_bytes();            // sizeof(Fp)
constexpr int TAB_CHUNK = 32;
void launch_table_windows(void *wb, const uint64_t *xext, int b0, int nb, int W, int cb, int prog_scale,
                          cudaStream_t st);
void launch_table_fill(uint4 *table, void *zs, const void *wb, int b0, int nb, int W, int cb, cudaStream_t st);
void launch_table_affine(uint4 *table, const void *zs, int b0, int nb, int W, int cb, cudaStream_t st);

// kernels_misc.cu
void launch_field_op(int field, int op, uint64_t *out, const uint64_t *a, const uint64_t *b, size_t count,
                     cudaStream_t st);
void launch_g1_op(int op, uint64_t *out, const uint64_t *a, const void *b, size_t count, cudaStream_t st);
void launch_fr_eq(uint8_t *eq, const uint64_t *x, const uint64_t *y, size_t count, cudaStream_t st);
void launch_g1p_eq(uint8_t *eq, const uint64_t *p, const uint64_t *q, size_t count, cudaStream_t st);
void launch_g1a_from_g1p(uint64_t *a, const uint64_t *p, size_t count, cudaStream_t st);
void launch_bench_field(int field, int sqr, uint32_t *data, size_t count, int iters, cudaStream_t st);
void launch_bench_imad(uint32_t *sink, int blocks, int threads, int iters, cudaStream_t st);
void launch_fingerprint(unsigned long long *out, const uint64_t *w, size_t n, cudaStream_t st);

inline unsigned blocks_for(size_t work, unsigned per) {
    size_t b = (work + per - 1) / per;
    return (unsigned)(b ? b : 1);
}
inline unsigned grid_stride_blocks(size_t work) {
    size_t b = (work + 255) / 256;
    return (unsigned)(b > 148 * 16 ? 148 * 16 : (b ? b : 1));
}

}  // namespace fk
