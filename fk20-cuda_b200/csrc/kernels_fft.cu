// kernels_fft.cu -- G1 FFT stages on row-interleaved tiles, and the
// reference <-> tile conversions.
//
// One warp per (butterfly, group of 32 rows): the twiddle of a butterfly is
// the same for all 32 rows, so its GLV/NAF program (scalar_prog.cuh) runs
// warp-uniformly.  The reference instead gives each thread a different
// butterfly of one row (g1p_fft.cu:25-177), so a 256-bit double-and-add per
// thread with divergent bits.  The two GLV base points of each thread live in
// a conflict-free shared-memory slot (word k of thread t at [k][t]).
// out-of-line Fp products for the stage kernels (see g1.cuh): their loops over
// point operations would otherwise not fit the instruction cache
#ifndef FK_FFT_OUTLINE
#define FK_FFT_OUTLINE 1
#endif
#if FK_FFT_OUTLINE
#define FK_FP_MUL_OUTLINE 1
#endif
#include "../../include/fk20_b200.h"
#include "check.cuh"
#include "consts.cuh"
#include "launch.h"
#include "layout.cuh"

#include <algorithm>

namespace fk {

cudaError_t upload_consts_fft() { return upload_module_consts(); }

FK_CHECK_WORD(fft)

// minimum resident blocks per SM requested from ptxas for the stage kernels
// (caps registers at 65536 / (FFT_THREADS * FK_FFT_MINB))
#ifndef FK_FFT_MINB
#define FK_FFT_MINB 1
#endif

// kind 0: DIF with inverse twiddles (natural in, bit-reversed out, no 1/m);
// kind 1: DIT with forward twiddles (bit-reversed in, natural out).
template <int KIND>
__global__ void __launch_bounds__(FFT_THREADS, FK_FFT_MINB) k_g1_stage(uint4 *__restrict__ D, int G, int log_m, int s) {
    __shared__ uint32_t slots[PROG_SLOT_WORDS][FFT_THREADS];
    const int m = 1 << log_m;
    const int warp = blockIdx.x * (FFT_THREADS / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    const int g = warp % G, b = warp / G;
    if (b >= (m >> 1)) return;
    int half, tix;
    if (KIND == 0) {
        half = m >> (s + 1);
        const int j = b & (half - 1);
        tix = ((m - (j << s)) << (MAX_LOG_M - log_m)) & 511;  // w_m^-(j 2^s) as a power of w_512
    } else {
        half = 1 << s;
        const int j = b & (half - 1);
        tix = (j << (log_m - 1 - s)) << (MAX_LOG_M - log_m);
    }
    const int j = b & (half - 1);
    const int i0 = ((b / half) * 2 * half) + j, i1 = i0 + half;
    uint4 *p0 = D + tile_index(g, m, i0);
    uint4 *p1 = D + tile_index(g, m, i1);
    const ProgSlots slot{&slots[0][threadIdx.x], FFT_THREADS};
    // Points pass through the shared-memory slots so that only the accumulator
    // of the current point operation is held in registers.
    G1P acc;
    if (KIND == 0) {
        // x = u + v, y = (u - v) * w^-t
        tile_to_slot(slot[0], p0, lane);
        tile_to_slot(slot[1], p1, lane);
        slot[0].load(acc);
        g1_add_q(acc, acc, slot[1], false);
        tile_store(p0, lane, acc);
        slot[0].load(acc);
        g1_add_q(acc, acc, slot[1], true);
        if (tix != 0) {
            slot[0].put(acc);
            g1_mul_prog(acc, slot, c_prog[tix]);
        }
        tile_store(p1, lane, acc);
    } else {
        // v' = v * w^t, x = u + v', y = u - v'
        tile_to_slot(slot[0], p1, lane);
        if (tix != 0) {
            g1_mul_prog(acc, slot, c_prog[tix]);
            slot[0].put(acc);
        }
        tile_to_slot(slot[1], p0, lane);
        slot[1].load(acc);
        g1_add_q(acc, acc, slot[0], false);
        tile_store(p0, lane, acc);
        slot[1].load(acc);
        g1_add_q(acc, acc, slot[0], true);
        tile_store(p1, lane, acc);
    }
}

// ------------------------------------------------------------------ fused stages
// One persistent launch runs the whole hext -> h_fft sequence of the plain
// pipeline -- inverse DIF stages 0..L-2, the middle stage, forward DIT stages
// 1..L-1 -- for every segment of the plan (segments may differ in length).
// Work is a stream of warp tasks (one butterfly of 32 rows) taken in order
// from a global counter; the stream is cut into blocks of (segment, stage) in
// stage-major order.  A task waits until the two positions it reads were
// written by the previous stage of its segment (per-position counters
// ready[g][i] = epoch * 64 + stage + 1, published with release semantics after
// the task's stores).  Tasks go only to running warps and a task only waits on
// tasks of lower index, so the lowest unfinished task never waits and every
// wait ends, also when not all blocks are resident.  The wait is still bounded
// (plan.spin_limit polls, default FUSED_SPIN_LIMIT): on expiry the kernel records an error code and
// returns instead of hanging.  Tile data written by other SMs is read through
// L2 (ld.cg) so no stale L1 line is used.

FK_D void tile_to_slot_cg(const StridedPoint &slot, const uint4 *base, int lane) {
#pragma unroll
    for (int q = 0; q < TILE_Q; q++) {
        const uint4 v = __ldcg(base + q * 32 + lane);
        slot.base[(4 * q) * slot.stride] = v.x;
        slot.base[(4 * q + 1) * slot.stride] = v.y;
        slot.base[(4 * q + 2) * slot.stride] = v.z;
        slot.base[(4 * q + 3) * slot.stride] = v.w;
    }
}

FK_D void tile_store_cg(uint4 *base, int lane, const G1P &p) {
    uint32_t w[36];
#pragma unroll
    for (int k = 0; k < 12; k++) { w[k] = p.x.w[k]; w[12 + k] = p.y.w[k]; w[24 + k] = p.z.w[k]; }
#pragma unroll
    for (int q = 0; q < TILE_Q; q++) __stcg(base + q * 32 + lane, make_uint4(w[4 * q], w[4 * q + 1], w[4 * q + 2], w[4 * q + 3]));
}

FK_D unsigned ld_acquire(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

FK_D void st_release(unsigned *p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// lane 0 waits until ready[a] and ready[b] reach `need`; false on timeout
FK_D bool wait_ready(const unsigned *ra, const unsigned *rb, unsigned need, int lane, unsigned limit) {
    int ok = 1;
    if (lane == 0) {
        unsigned spins = 0;
        while (ld_acquire(ra) < need || ld_acquire(rb) < need) {
            if (++spins >= limit) { ok = 0; break; }
            __nanosleep(64);
        }
    }
    ok = __shfl_sync(0xffffffffu, ok, 0);
    __threadfence();
    return ok != 0;
}

__global__ void __launch_bounds__(FFT_THREADS, FK_FFT_MINB) k_g1_fused(const __grid_constant__ FusedPlan P) {
    __shared__ uint32_t slots[PROG_SLOT_WORDS][FFT_THREADS];
    const int lane = threadIdx.x & 31;
    const unsigned total = P.blk.start[P.blk.nblk];
    const unsigned base = P.epoch * 64u;
    const ProgSlots slot{&slots[0][threadIdx.x], FFT_THREADS};
    for (;;) {
        unsigned task = 0;
        if (lane == 0) task = atomicAdd(P.next, 1u);
        task = __shfl_sync(0xffffffffu, task, 0);
        if (task >= total) return;
        if (*(volatile int *)P.err) return;
        FusedTask t;
        fused_task_decode(t, P.blk, task);
        // checked build: the decoded task lies in its segment and names a
        // program; otherwise stop the launch (no access, no publication)
        if (!FK_CHECK(g_check_fft, t.seg >= 0 && t.seg < P.blk.nseg && t.g >= 0 && t.g < P.blk.G[t.seg] &&
                                       t.i0 >= 0 && t.i1 < (1 << P.blk.log_m[t.seg]) && t.i0 < t.i1,
                      FK20_CHECK_FFT_TASK) ||
            !FK_CHECK(g_check_fft, t.tix >= 0 && t.tix < NPROG, FK20_CHECK_FFT_PROGRAM)) {
            if (lane == 0) atomicCAS(P.err, 0, 2000);
            return;
        }
        const FusedSeg &a = P.seg[t.seg];
        const int m = 1 << P.blk.log_m[t.seg];
        const int S = t.S, g = t.g, i0 = t.i0, i1 = t.i1, tix = t.tix, kind = t.kind;
        unsigned *r0 = a.ready + (size_t)g * m + i0, *r1 = a.ready + (size_t)g * m + i1;
        if (S > 0 && !wait_ready(r0, r1, base + (unsigned)S, lane, P.spin_limit)) {
            if (lane == 0) atomicCAS(P.err, 0, 1000 + S);
            return;
        }
        uint4 *p0 = a.D + tile_index(g, m, i0);
        uint4 *p1 = a.D + tile_index(g, m, i1);
        G1P acc;
        if (kind == 0) {
            tile_to_slot_cg(slot[0], p0, lane);
            tile_to_slot_cg(slot[1], p1, lane);
            slot[0].load(acc);
            g1_add_q(acc, acc, slot[1], false);
            tile_store_cg(p0, lane, acc);
            slot[0].load(acc);
            g1_add_q(acc, acc, slot[1], true);
            if (tix != 0) {
                slot[0].put(acc);
                g1_mul_prog(acc, slot, c_prog[tix]);
            }
            tile_store_cg(p1, lane, acc);
        } else if (kind == 2) {
            tile_to_slot_cg(slot[1], p1, lane);
            tile_to_slot_cg(slot[0], p0, lane);
            slot[0].load(acc);
            g1_add_q(acc, acc, slot[1], false);
            tile_store_cg(p0, lane, acc);
            tile_store_cg(p1, lane, acc);
        } else {
            tile_to_slot_cg(slot[0], p1, lane);
            if (tix != 0) {
                g1_mul_prog(acc, slot, c_prog[tix]);
                slot[0].put(acc);
            }
            tile_to_slot_cg(slot[1], p0, lane);
            slot[1].load(acc);
            g1_add_q(acc, acc, slot[0], false);
            tile_store_cg(p0, lane, acc);
            slot[1].load(acc);
            g1_add_q(acc, acc, slot[0], true);
            tile_store_cg(p1, lane, acc);
        }
        __threadfence();
        __syncwarp();
        if (lane == 0) {
            if (task != P.unpublished) {  // see FusedPlan::unpublished (tests of the bounded wait)
                st_release(r0, base + (unsigned)S + 1u);
                st_release(r1, base + (unsigned)S + 1u);
            }
        }
    }
}

int fused_blocks_per_sm() {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_g1_fused, FFT_THREADS, 0) != cudaSuccess) return 0;
    return n;
}

void launch_g1_fused(const FusedPlan &p, cudaStream_t st) {
    k_g1_fused<<<p.blocks, FFT_THREADS, 0, st>>>(p);
}

// last DIF stage + zeroing of the upper half + first DIT stage: pairs
// (2q, 2q+1) -> both = a + b, optionally times 2^-log_m
template <bool SCALE>
__global__ void __launch_bounds__(FFT_THREADS) k_g1_middle(uint4 *__restrict__ D, int G, int log_m) {
    // the program scratch (SCALE), whose point 1 also holds b for the sum;
    // without SCALE one point of scratch
    __shared__ uint32_t slots[SCALE ? PROG_SLOT_WORDS : 36][FFT_THREADS];
    const int m = 1 << log_m;
    const int warp = blockIdx.x * (FFT_THREADS / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    const int g = warp % G, q = warp / G;
    if (q >= (m >> 1)) return;
    uint4 *p0 = D + tile_index(g, m, 2 * q);
    uint4 *p1 = D + tile_index(g, m, 2 * q + 1);
    const StridedPoint sv{&slots[SCALE ? 36 : 0][threadIdx.x], FFT_THREADS};
    G1P x;
    tile_to_slot(sv, p1, lane);
    tile_load(x, p0, lane);
    g1_add_q(x, x, sv, false);
    if (SCALE) {
        const ProgSlots slot{&slots[0][threadIdx.x], FFT_THREADS};
        slot[0].put(x);
        g1_mul_prog(x, slot, c_prog[512 + log_m]);
    }
    tile_store(p0, lane, x);
    tile_store(p1, lane, x);
}

// every point of the tiles times program `prog`
__global__ void __launch_bounds__(FFT_THREADS) k_g1_scale(uint4 *__restrict__ D, int G, int log_m, int prog) {
    __shared__ uint32_t slots[PROG_SLOT_WORDS][FFT_THREADS];
    const int m = 1 << log_m;
    const int warp = blockIdx.x * (FFT_THREADS / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    const int g = warp % G, i = warp / G;
    if (i >= m) return;
    uint4 *p = D + tile_index(g, m, i);
    const ProgSlots slot{&slots[0][threadIdx.x], FFT_THREADS};
    G1P u;
    tile_to_slot(slot[0], p, lane);
    g1_mul_prog(u, slot, c_prog[prog]);
    tile_store(p, lane, u);
}

// reference g1p_t rows [rows][m] -> tiles.  bitrev_in: element i goes to
// position bitrev(i); zero_upper: elements i >= m/2 taken as infinity.
// Lanes of padding rows hold infinity.
__global__ void k_ref_to_tile(uint4 *__restrict__ D, const uint64_t *__restrict__ src, int rows, int G, int log_m,
                              int bitrev_in, int zero_upper) {
    const int m = 1 << log_m;
    const size_t total = (size_t)G * 32 * m;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int row = (int)(e / m), i = (int)(e % m);
        G1P p;
        if (row < rows && !(zero_upper && i >= (m >> 1))) g1p_from_ref(p, src + 18 * e);
        else g1_set_inf(p);
        const int pos = bitrev_in ? (int)bitrev((unsigned)i, log_m) : i;
        tile_store(D + tile_index(row >> 5, m, pos), row & 31, p);
    }
}

// tiles -> reference g1p_t rows, natural order; row r is written at
// dst + 18 * (row_off ? row_off[r] : r * m)
__global__ void k_tile_to_ref(uint64_t *__restrict__ dst, const uint4 *__restrict__ D, const size_t *__restrict__ row_off,
                              int rows, int log_m, int bitrev_out) {
    const int m = 1 << log_m;
    const size_t total = (size_t)rows * m;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int row = (int)(e / m), i = (int)(e % m);
        const int pos = bitrev_out ? (int)bitrev((unsigned)i, log_m) : i;
        G1P p;
        tile_load(p, D + tile_index(row >> 5, m, pos), row & 31);
        const size_t base = row_off ? row_off[row] : (size_t)row * m;
        g1p_to_ref(dst + 18 * (base + i), p);
    }
}

// h[row][m/2 .. m-1] = infinity, in place (fk20_hext2h, fk20_poly2h_fft.cu:27-33)
__global__ void k_hext2h_ref(uint64_t *__restrict__ h, int rows, int log_m) {
    const int m = 1 << log_m;
    const size_t total = (size_t)rows * (m >> 1);
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const size_t row = e / (m >> 1), i = (m >> 1) + e % (m >> 1);
        uint64_t *gp = h + 18 * (row * m + i);
#pragma unroll
        for (int k = 0; k < 18; k++) gp[k] = 0;
        gp[6] = 1;
    }
}

// setup -> bit-reversed FFT input tiles for xext_fft: lane i < 16, position j:
// x_j = setup[n - l - 1 - i - l j] for j < k - 1, else infinity
// (FK20Py/fk20_multi_cuda.py:104-109, fk20_single.py:45-58)
__global__ void k_setup_to_tile(uint4 *D, const uint64_t *setup, int n, int log_m) {
    const int m = 1 << log_m;
    const int k = n / L_COLS;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < 32 * m; e += gridDim.x * blockDim.x) {
        const int lane = e / m, j = e % m;
        G1P p;
        if (lane < L_COLS && j < k - 1) g1p_from_ref(p, setup + 18 * (size_t)(n - L_COLS - 1 - lane - L_COLS * j));
        else g1_set_inf(p);
        tile_store(D + tile_index(0, m, (int)bitrev((unsigned)j, log_m)), lane, p);
    }
}

void launch_g1_stage(uint4 *D, int G, int log_m, int s, int kind, cudaStream_t st) {
    const unsigned blocks = blocks_for((size_t)G * ((1u << log_m) / 2), FFT_THREADS / 32);
    if (kind == 0) k_g1_stage<0><<<blocks, FFT_THREADS, 0, st>>>(D, G, log_m, s);
    else k_g1_stage<1><<<blocks, FFT_THREADS, 0, st>>>(D, G, log_m, s);
}
void launch_g1_middle(uint4 *D, int G, int log_m, int scale, cudaStream_t st) {
    const unsigned blocks = blocks_for((size_t)G * ((1u << log_m) / 2), FFT_THREADS / 32);
    if (scale) k_g1_middle<true><<<blocks, FFT_THREADS, 0, st>>>(D, G, log_m);
    else k_g1_middle<false><<<blocks, FFT_THREADS, 0, st>>>(D, G, log_m);
}
void launch_g1_scale(uint4 *D, int G, int log_m, int prog, cudaStream_t st) {
    k_g1_scale<<<blocks_for((size_t)G * (1u << log_m), FFT_THREADS / 32), FFT_THREADS, 0, st>>>(D, G, log_m, prog);
}
void launch_ref_to_tile(uint4 *D, const uint64_t *src, int rows, int G, int log_m, int bitrev_in, int zero_upper,
                        cudaStream_t st) {
    k_ref_to_tile<<<grid_stride_blocks((size_t)G * 32 * (1u << log_m)), 256, 0, st>>>(D, src, rows, G, log_m,
                                                                                   bitrev_in, zero_upper);
}
void launch_tile_to_ref(uint64_t *dst, const uint4 *D, const size_t *row_off, int rows, int log_m, int bitrev_out,
                        cudaStream_t st) {
    k_tile_to_ref<<<grid_stride_blocks((size_t)rows << log_m), 256, 0, st>>>(dst, D, row_off, rows, log_m, bitrev_out);
}
void launch_hext2h_ref(uint64_t *h, int rows, int log_m, cudaStream_t st) {
    k_hext2h_ref<<<grid_stride_blocks((size_t)rows << (log_m - 1)), 256, 0, st>>>(h, rows, log_m);
}
void launch_setup_to_tile(uint4 *D, const uint64_t *setup, int n, int log_m, cudaStream_t st) {
    k_setup_to_tile<<<grid_stride_blocks((size_t)32 << log_m), 256, 0, st>>>(D, setup, n, log_m);
}

}  // namespace fk
