// fused_plan.cuh -- task numbering of the persistent stage-fused G1 FFT
// (kernels_fft.cu k_g1_fused).  Host and device code: the engine builds the
// block table, the kernel decodes tasks with it, and the CPU tests check the
// schedule's properties with the same functions.
//
// A plan covers up to MAX_SEGS segments (FK20 instances of one length each,
// G row groups of 32 at FFT size m = 2^log_m).  Segment k runs 2 log_m - 1
// stages: inverse DIF stages 0..log_m-2, the middle stage (last inverse
// butterfly + zeroing of the upper half + first forward butterfly), forward
// DIT stages 1..log_m-1.  Each stage is G * m/2 warp tasks (one butterfly of
// 32 rows).  The task stream is cut into blocks (segment, stage) in
// stage-major order, so every task of stage S > 0 only reads positions that
// tasks of lower index wrote at stage S - 1.
#pragma once
#include "limbs.cuh"

namespace fk {

constexpr int MAX_SEGS = 24;
constexpr int FUSED_MAX_LOG_M = 9;
constexpr int MAX_FUSED_STAGES = 2 * FUSED_MAX_LOG_M - 1;
constexpr int MAX_FUSED_BLOCKS = MAX_SEGS * MAX_FUSED_STAGES;

struct FusedBlocks {
    unsigned start[MAX_FUSED_BLOCKS + 1];  // first task of each block; [nblk] = task count
    unsigned char seg[MAX_FUSED_BLOCKS], stage[MAX_FUSED_BLOCKS];
    int nblk;
    int G[MAX_SEGS], log_m[MAX_SEGS];
    // stage window [s_lo, s_hi) of each segment; s_hi = 0 means all its
    // stages.  A segment whose window starts above stage 0 continues the
    // stages an earlier launch ran on the same tiles and readiness counters
    // (counters kept, same epoch), so its first stage finds its inputs ready.
    unsigned char s_lo[MAX_SEGS], s_hi[MAX_SEGS];
    int nseg;
};

FK_HD int fused_stage_hi(const FusedBlocks &b, int k) { return b.s_hi[k] ? b.s_hi[k] : 2 * b.log_m[k] - 1; }

// fills start/seg/stage from G, log_m, nseg; returns the task count
// Blocks go in order of the stage RELATIVE to each segment's window (its
// first stage in this launch, then its second, ...): segments whose windows
// start at different stages then progress side by side, and a launch lasts
// about as many task times as its longest window, not the span of all
// windows.  A task of relative stage r only reads what tasks of relative
// stage r - 1 of its own segment (lower task indices) or an earlier launch
// wrote.
FK_HD unsigned fused_blocks_build(FusedBlocks &b) {
    int maxw = 0;
    for (int k = 0; k < b.nseg; k++)
        if (fused_stage_hi(b, k) - b.s_lo[k] > maxw) maxw = fused_stage_hi(b, k) - b.s_lo[k];
    unsigned task = 0;
    int nb = 0;
    for (int r = 0; r < maxw; r++)
        for (int k = 0; k < b.nseg; k++) {
            const int S = b.s_lo[k] + r;
            if (S >= fused_stage_hi(b, k)) continue;
            b.start[nb] = task;
            b.seg[nb] = (unsigned char)k;
            b.stage[nb] = (unsigned char)S;
            nb++;
            task += (unsigned)b.G[k] * ((1u << b.log_m[k]) >> 1);
        }
    b.nblk = nb;
    b.start[nb] = task;
    return task;
}

struct FusedTask {
    int seg, S, g;
    int i0, i1;  // positions (in the segment's tile of group g) the butterfly reads and writes
    int tix;     // twiddle as a power of w_512 (0: none)
    int kind;    // 0 inverse DIF, 1 forward DIT, 2 middle
};

// task < b.start[b.nblk]
FK_HD void fused_task_decode(FusedTask &t, const FusedBlocks &b, unsigned task) {
    int lo = 0, hi = b.nblk - 1;  // the last block with start <= task
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (b.start[mid] <= task) lo = mid;
        else hi = mid - 1;
    }
    t.seg = b.seg[lo];
    t.S = b.stage[lo];
    const int L = b.log_m[t.seg], m = 1 << L, G = b.G[t.seg];
    const int r = (int)(task - b.start[lo]);
    t.g = r % G;
    const int bf = r / G;
    t.tix = 0;
    if (t.S < L - 1) {  // inverse DIF stage s = S: pairs (i, i + m/2^(s+1)), twiddle w_m^-(j 2^s)
        t.kind = 0;
        const int half = m >> (t.S + 1), j = bf & (half - 1);
        t.i0 = (bf / half) * 2 * half + j;
        t.i1 = t.i0 + half;
        t.tix = ((m - (j << t.S)) << (FUSED_MAX_LOG_M - L)) & 511;
    } else if (t.S == L - 1) {  // middle: pairs (2q, 2q + 1)
        t.kind = 2;
        t.i0 = 2 * bf;
        t.i1 = 2 * bf + 1;
    } else {  // forward DIT stage s = S - L + 1: pairs (i, i + 2^s), twiddle w_m^(j m / 2^(s+1))
        t.kind = 1;
        const int s = t.S - L + 1, half = 1 << s, j = bf & (half - 1);
        t.i0 = (bf / half) * 2 * half + j;
        t.i1 = t.i0 + half;
        t.tix = (j << (L - 1 - s)) << (FUSED_MAX_LOG_M - L);
    }
}

}  // namespace fk
