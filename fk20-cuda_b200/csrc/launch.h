// launch.h -- host launchers exported by the kernel translation units.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "fused_plan.cuh"

namespace fk {

constexpr int FFT_THREADS = 64;  // threads per block of the G1 FFT stage kernels
constexpr int FFT_WARPS = FFT_THREADS / 32;

// A launch may cover several segments (fused_plan.cuh): runs of FK20
// instances of one length each; a ragged batch has one per length.

// fixed-base MSM over the segments' scalar tiles S into their point tiles D
struct MsmSeg {
    uint4 *D;
    const uint4 *S;
    const uint4 *table;
    int G, log_m, rows, cb, W;
    unsigned warp_start;  // first warp (of the launch) that works on this segment
};
struct MsmArgs {
    MsmSeg seg[MAX_SEGS];
    int nseg, times_m;
    int test_check;  // checked build: record FK20_CHECK_MSM_PLANTED (tests of the checks)
    unsigned warps;  // total warps = sum of G * m
};

// Persistent stage-fused G1 FFT plan: the segments' tiles and readiness
// counters, and the task block table (fused_plan.cuh).
struct FusedSeg {
    uint4 *D;
    unsigned *ready;  // [G][m] readiness counters of this segment
};
struct FusedPlan {
    FusedSeg seg[MAX_SEGS];
    FusedBlocks blk;
    unsigned *next;  // task counter (zeroed before the launch)
    int *err;        // 0 = ok, else 1000 + stage that timed out
    unsigned epoch;  // readiness value base (epoch * 64 + stage + 1), < 2^26
    int blocks;      // grid size: resident blocks of the persistent launch
    unsigned spin_limit;   // polls before a readiness wait gives up
    // A task whose completion is not published (0xffffffff: none).  Set only
    // by tests of the bounded wait: the tasks that read its positions wait
    // until spin_limit, and the launch ends with the error flag set.
    unsigned unpublished;
};
constexpr unsigned FUSED_SPIN_LIMIT = 1u << 24;  // default spin_limit

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
void launch_msm(const MsmArgs &a, int threads, cudaStream_t st);  // threads: 64, 128 or 256
// checked build (check.cuh): take and clear the first failing check site of the
// MSM / persistent-FFT translation units (0: none)
int check_take_msm();
int check_take_fft();
// KZG commitments: polynomial lengths are multiples of COMMIT_CHUNK; pass 1
// has commit_parts(rows, n) warps per 32 rows, and part holds as many tiles
constexpr int COMMIT_CHUNK = 32;
int commit_parts(int rows, int n);
void launch_commit(uint64_t *out, uint4 *part, const uint64_t *poly, const uint4 *table, int rows, int n, int W,
                   int cb, cudaStream_t st);

// kernels_fft.cu
void launch_g1_stage(uint4 *D, int G, int log_m, int s, int kind, cudaStream_t st);
void launch_g1_middle(uint4 *D, int G, int log_m, int scale, cudaStream_t st);
int fused_blocks_per_sm();
void launch_g1_fused(const FusedPlan &p, cudaStream_t st);
void launch_g1_scale(uint4 *D, int G, int log_m, int prog, cudaStream_t st);
void launch_ref_to_tile(uint4 *D, const uint64_t *src, int rows, int G, int log_m, int bitrev_in, int zero_upper,
                        cudaStream_t st);
void launch_tile_to_ref(uint64_t *dst, const uint4 *D, const size_t *row_off, int rows, int log_m, int bitrev_out,
                        cudaStream_t st);
void launch_hext2h_ref(uint64_t *h, int rows, int log_m, cudaStream_t st);
void launch_setup_to_tile(uint4 *D, const uint64_t *setup, int n, int log_m, cudaStream_t st);

// kernels_out.cu: 48-byte compressed proofs, data-availability order
void launch_g1p_compress(uint8_t *out, const uint64_t *p, size_t count, cudaStream_t st);
void launch_h_fft_to_proofs(uint8_t *out, const uint64_t *h, int rows, int log_m, cudaStream_t st);
void launch_tile_to_proofs(uint8_t *out, const uint4 *D, const size_t *out_off, int rows, int log_m,
                           cudaStream_t st);

// kernels_pairing.cu: op 0 pairing values, op 1 pairing checks; G2 element-wise ops
void launch_pairing(int op, uint64_t *out, uint8_t *ok, const uint64_t *a, const uint64_t *b, const uint64_t *c,
                    const uint64_t *d, size_t count, cudaStream_t st, int bcast = 0);
void launch_interp(uint64_t *poly, uint64_t *xl, const uint64_t *x, const uint64_t *ys, int log_l, size_t count,
                   cudaStream_t st);
void launch_g2_op(int op, uint64_t *out, const uint64_t *a, const void *b, size_t count, cudaStream_t st);

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
