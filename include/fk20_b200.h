/*
 * fk20_b200.h -- C ABI of the B200 FK20 engine (libfk20b200.so).
 *
 * Drop-in for the FK20 hot path of lCardosoSantos/FK20-CUDA: every amortized
 * KZG proof of a batch of polynomials against one shared setup.  Entry-point
 * names and argument meanings follow the reference (fk20.cuh:20-38,
 * fr.cuh:62-69, g1.cuh:98-108); the reference's __global__ kernels, which a
 * caller launched with <<<rows, 256, smem>>>, become host launchers here.
 *
 * Conventions (all entry points):
 *  - Buffers are DEVICE pointers in the reference layouts: fr_t = 4 x uint64,
 *    fp_t = 6 x uint64, g1p_t = {x, y, z} homogeneous projective (x = X/Z,
 *    y = Y/Z), little-endian, standard (non-Montgomery) form.  Inputs may be
 *    any representative (fp_t < 2^384, fr_t < 2^256, like the reference);
 *    outputs are canonical (< p, < r), and a point at infinity is written as
 *    (0, 1, 0) (g1p.cu:95-100).  G1 inputs must lie in the order-r subgroup
 *    (true of every FK20 value: setup multiples and their combinations).
 *  - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream);
 *    work is enqueued asynchronously, like the reference's launches.
 *  - Return value: 0 on success, a cudaError_t value (1..999) for a CUDA
 *    failure, or one of the FK20_E* codes below for a rejected argument.
 *    Nothing traps; arguments are validated on the host before any launch.
 *  - The l = 16 chunking of the reference is fixed; polynomial length
 *    n in {1024, 2048, 4096} gives FFT size m = 2n/16 in {128, 256, 512}.
 *    The reference entry points without an `n` argument use n = 4096, m = 512.
 */
#ifndef FK20_B200_H
#define FK20_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef uint64_t fr_t[4];
typedef uint64_t fp_t[6];
typedef struct { fp_t x, y; } g1a_t;
typedef struct { fp_t x, y, z; } g1p_t;

#define FK20_OK 0
#define FK20_EINVAL 1001   /* bad size, row count, null pointer or alignment */
#define FK20_ENOSETUP 1002 /* context has no tables for this polynomial length */
#define FK20_ENOMEM 1003   /* device allocation failed */
#define FK20_ENODEV 1004   /* no usable sm_100 device */
#define FK20_ETIMEOUT 1005 /* a persistent launch gave up waiting (results invalid) */
#define FK20_ETOOBIG 1006  /* request larger than the fixed scratch of a no-allocation entry point */
#define FK20_EAGAIN 1007   /* server: the request is not finished yet / the queue is full */
#define FK20_ECHECK 1008   /* checked build: a kernel check stopped a launch (fk20_check_status says which) */
#define FK20_ECANCELED 1009 /* server: the request was cancelled before it was packed */

/* ------------------------------------------------------------------ context
 * A context owns, on one device, the fixed-base tables built from xext_fft
 * (one set per polynomial length) and the per-call workspaces.  Calls on one
 * context are serialised by an internal lock and run in stream order; use one
 * context per concurrent stream.  No reference counterpart: the reference keeps
 * this state in file-scope __managed__ arrays (fk20_poly2h_fft.cu:15-16,
 * fk20_msm.cu:357-360), which is why it is not re-entrant.
 */
typedef struct fk20_ctx fk20_ctx;

/* window: signed-digit width of the fixed-base tables (8..15; 0 = default 10).
 * The MSM splits each scalar s = s1 + s2 lambda with the GLV endomorphism
 * (s1, s2 < 2^128), so the tables cover 129-bit digits: bytes per polynomial
 * length n: 16*m bases * ceil(129/w) windows * 2^(w-1) entries * 96 B
 * (5.2 GB for n = 4096, w = 10; 116 GB at w = 15).  The default context
 * behind the reference-signature entry points takes its window from the
 * environment variable FK20_WINDOW (read once per device), else 10. */
int fk20_ctx_create(fk20_ctx **ctx, int device, int window);
int fk20_ctx_destroy(fk20_ctx *ctx);

/* Build the tables of length n from xext_fft[16][m] (device, g1p_t).
 * Replaces fk20_msm_makelut (fk20_msm.cu:79-141). */
int fk20_ctx_load_xext_fft(fk20_ctx *ctx, unsigned n, const g1p_t *xext_fft, void *stream);

/* xext_fft[16][m] from the setup s_0..s_{n-1} (device g1p_t) on the GPU, then
 * build the tables.  Replaces the reference's fk20_setup2xext_fft (fk20.cu:28-59,
 * which its own comment marks as failing) and the Python precompute
 * FK20Py/fk20_multi_cuda.py:104-109. */
int fk20_ctx_load_setup(fk20_ctx *ctx, unsigned n, const g1p_t *setup, void *stream);

/* h_fft[rows][m] (the m = 2n/16 proofs of each row) for rows x n polynomial
 * coefficients, against the context's tables for n.  Same computation as the
 * reference's host pipeline fk20_poly2h_fft (fk20_poly2h_fft.cu:47-78). */
int fk20_ctx_poly2h_fft(fk20_ctx *ctx, g1p_t *h_fft, const fr_t *polynomial, unsigned rows, unsigned n,
                        void *stream);

/* Same, with intermediate hext_fft[rows][m] also written (may be NULL). */
int fk20_ctx_poly2hext_fft(fk20_ctx *ctx, g1p_t *hext_fft, const fr_t *polynomial, unsigned rows, unsigned n,
                           void *stream);

/* MSM stage alone: hext_fft[rows][m] = sum_i tc_fft[row][i][c] * xext_fft[i][c]
 * for tc_fft[rows][16][m] (fk20_msm.cu:23-66). */
int fk20_ctx_msm(fk20_ctx *ctx, g1p_t *hext_fft, const fr_t *tc_fft, unsigned rows, unsigned n, void *stream);

/* Ragged batch: `count` independent FK20 instances, instance j with length
 * n_j in {1024, 2048, 4096}, polynomial at poly_off[j] (in fr_t units from
 * `polys`) and m_j proofs written at out_off[j] (in g1p_t units from `h_fft`).
 * All offset arrays are HOST arrays (read before the call returns).  The
 * instances are grouped into one segment per length, and all segments run in
 * ONE fixed-base MSM launch and ONE persistent stage-fused G1 FFT launch.
 * No reference counterpart (the reference proves one length per call). */
int fk20_ctx_batch(fk20_ctx *ctx, g1p_t *h_fft, const fr_t *polys, unsigned count, const unsigned *n,
                   const size_t *poly_off, const size_t *out_off, void *stream);

/* Batch plan: a fixed ragged batch layout (the arguments of fk20_ctx_batch)
 * bound to fixed device buffers, captured once into a CUDA graph with its own
 * workspace; fk20_plan_launch replays the whole batch as one graph launch.
 * Launches of one plan must be stream-ordered (they share its workspace).  A
 * plan whose tables were rebuilt since its creation (reload, autotune)
 * returns FK20_ENOSETUP; fk20_plan_launch returns FK20_ETIMEOUT once a
 * replay's persistent launch gave up.  No reference counterpart. */
typedef struct fk20_plan fk20_plan;
int fk20_plan_create(fk20_plan **plan, fk20_ctx *ctx, g1p_t *h_fft, const fr_t *polys, unsigned count,
                     const unsigned *n, const size_t *poly_off, const size_t *out_off);
int fk20_plan_launch(fk20_plan *plan, void *stream);
int fk20_plan_destroy(fk20_plan *plan);

/* Autotuner (no reference counterpart): times the pipeline for length n on
 * `rows` seeded sample rows under each candidate -- table window 8..15 whose
 * tables fit in max_table_bytes (0 = what the free device memory allows),
 * MSM block size 64/128/256, persistent FFT grid 1..max blocks per SM, fused
 * or staged FFT -- one parameter at a time, keeps the fastest in the context
 * (tables rebuilt at the chosen window) and reports it.  Needs the tables of
 * n loaded.  Synchronous; takes seconds (one table build per window). */
typedef struct {
    int window, msm_threads, fft_blocks_per_sm, fused_fft;
    float ms;          /* best time for `rows` rows */
    float ms_default;  /* time of the configuration the context had before */
} fk20_tune_result;
int fk20_ctx_autotune(fk20_ctx *ctx, unsigned n, unsigned rows, size_t max_table_bytes, fk20_tune_result *result,
                      void *stream);

/* Options.  FK20_OPT_FUSED_FFT (default 1): run the inverse and forward G1
 * FFT stages of the pipeline as one persistent launch whose warps take
 * butterfly tasks in stage order and wait (bounded) for their inputs, instead
 * of one launch per stage. */
#define FK20_OPT_FUSED_FFT 1
/* FK20_OPT_MSM_THREADS: MSM block size, 64, 128 (default) or 256 threads. */
#define FK20_OPT_MSM_THREADS 2
/* FK20_OPT_FFT_BLOCKS_PER_SM: persistent FFT grid, blocks per SM (0 =
 * default: as many as fit). */
#define FK20_OPT_FFT_BLOCKS_PER_SM 3
/* FK20_OPT_WAIT_LIMIT: polls a readiness wait of the persistent FFT makes
 * before it gives up and the launch reports FK20_ETIMEOUT (0 = default 2^24). */
#define FK20_OPT_WAIT_LIMIT 4
/* FK20_OPT_TEST_UNPUBLISHED_TASK: for tests of that bounded wait only -- the
 * task of this index in the next persistent launches never publishes its
 * completion, so the tasks that read its outputs wait until the limit and
 * the call's results are invalid (fk20_ctx_status returns FK20_ETIMEOUT and
 * clears the condition).  -1 (default) = off. */
#define FK20_OPT_TEST_UNPUBLISHED_TASK 5
/* FK20_OPT_WINDOW: table window (8..15) of the tables that later
 * fk20_ctx_load_setup / fk20_ctx_load_xext_fft calls build (tables already
 * built keep theirs), so each polynomial length can have its own: tables of
 * length n hold 2n (ceil(129 / w)) 2^(w-1) entries of 96 bytes -- at n = 4096,
 * 32 GB at w = 13 and 116 GB at w = 15 (9 instead of 10 windows per GLV
 * half). */
#define FK20_OPT_WINDOW 6
/* FK20_OPT_TEST_CHECK: for tests of the checked build only -- nonzero makes
 * the next MSM launches record FK20_CHECK_MSM_PLANTED (the normal build
 * ignores it). */
#define FK20_OPT_TEST_CHECK 7
int fk20_ctx_set(fk20_ctx *ctx, int option, int value);
int fk20_ctx_get(fk20_ctx *ctx, int option, int *value);

/* Waits for the context's queued work; returns FK20_ETIMEOUT if a persistent
 * launch gave up waiting (its outputs are then invalid), else 0 or a CUDA
 * error.  Bounded waits, not traps: the device context stays usable. */
int fk20_ctx_status(fk20_ctx *ctx);

/* Device bytes the context holds (tables + workspaces). */
size_t fk20_ctx_device_bytes(const fk20_ctx *ctx);

/* Per-launch profiling (no reference counterpart; the reference times whole
 * calls with cudaEvents in fk20benchmark.cu:103-116).  While enabled, every
 * pipeline kernel a call on this context launches is bracketed by CUDA events
 * on its stream and tagged with its work in 32x32->64-bit limb products.
 * fk20_ctx_profile(ctx, 1) resets the totals and enables;
 * fk20_ctx_profile_read waits for the recorded launches and returns the totals
 * of one kernel kind, its work counted ALGORITHMICALLY: an Fp product or
 * square 300 limb products, an Fr product 136, a G1 addition 12, mixed
 * addition 11 and doubling 8 Fp products, a fixed-scalar multiplication its
 * chain's doublings and additions at those prices (the work the roofline
 * fraction divides by, whatever formulas a kernel uses).
 * fk20_ctx_profile_read_executed returns the same kind's work as EXECUTED by
 * the kernels' cheaper formulas (triangular squares of 234, XYZZ mixed
 * additions of 8 M + 2 S, Jacobian twiddle programs on an isomorphic curve). */
#define FK20_K_TC_FFT 0    /* toeplitz + Fr FFTs */
#define FK20_K_MSM 1       /* fixed-base MSM */
#define FK20_K_STAGE_INV 2 /* inverse G1 FFT stages */
#define FK20_K_STAGE_FWD 3 /* forward G1 FFT stages */
#define FK20_K_MIDDLE 4    /* last inverse + zeroing + first forward stage */
#define FK20_K_OUTPUT 5    /* tiles -> reference g1p_t */
#define FK20_K_FFT_FUSED 6 /* all G1 FFT stages in one persistent launch */
#define FK20_NKINDS 7
int fk20_ctx_profile(fk20_ctx *ctx, int enable);
int fk20_ctx_profile_read(fk20_ctx *ctx, int kind, double *ms, long *launches, double *products);
int fk20_ctx_profile_read_executed(fk20_ctx *ctx, int kind, double *products);

/* Doublings and additions of the fixed-scalar G1 program `index` (0..511:
 * w_512^index; 512 + s: 2^-s), for work accounting. */
int fk20_program_cost(int index, int *dbl, int *add);

/* ------------------------------------------------------------------ KZG commitments
 * commitment[r] = sum_i polynomial[r][i] * s_i, the commitment of
 * commit_to_poly (FK20Py/kzg_proofs.py:159-163; no CUDA counterpart in the
 * reference), as a fixed-base MSM over tables of the setup points s_0..s_{n-1}:
 * fk20_ctx_load_commit builds them (window 8..13, 0 = 10; n a multiple of 32,
 * at most 65536: 4096 points at window 10 take 5.2 GB), fk20_ctx_commit
 * commits rows polynomials of n' <= n coefficients (n' a multiple of 32). */
int fk20_ctx_load_commit(fk20_ctx *ctx, unsigned n, const g1p_t *setup, int window, void *stream);
int fk20_ctx_commit(fk20_ctx *ctx, g1p_t *commitment, const fr_t *polynomial, unsigned rows, unsigned n,
                    void *stream);

/* ------------------------------------------------------------------ data-availability output
 * Proofs as data-availability consumers read them (no CUDA counterpart in the
 * reference; the Python path is FK20Py/fk20_multi_cuda.py:249-260 with
 * list_to_reverse_bit_order, FK20Py/kzg_proofs.py:105-118): each proof is the
 * 48-byte compressed encoding of its affine point -- x big-endian, flag bits
 * 0x80 compressed, 0x40 infinity, 0x20 y > (p-1)/2 in the first byte -- and the
 * m proofs of a row are in bit-reversed order: proof i of a row is
 * h_fft[bitrev(i)].  Output buffers are DEVICE bytes, 16-byte aligned. */

/* out[count][48] = compressed encodings of p[count] (natural order) */
int fk20_g1p_compress_n(uint8_t *out, const g1p_t *p, size_t count, void *stream);

/* h_fft[rows][m] -> proofs[rows][m][48] in data-availability order */
int fk20_h_fft2proofs(uint8_t *proofs, const g1p_t *h_fft, unsigned rows, unsigned n, void *stream);

/* The whole pipeline with this output written straight from the engine's
 * tiles: polynomial[rows][n] -> proofs[rows][m][48]. */
int fk20_ctx_poly2proofs(fk20_ctx *ctx, uint8_t *proofs, const fr_t *polynomial, unsigned rows, unsigned n,
                         void *stream);

/* Ragged batch (as fk20_ctx_batch) with this output; out_off[j] counts proofs. */
int fk20_ctx_batch_proofs(fk20_ctx *ctx, uint8_t *proofs, const fr_t *polys, unsigned count, const unsigned *n,
                          const size_t *poly_off, const size_t *out_off, void *stream);

/* ------------------------------------------------------------------ pairings (proof verification)
 * BLS12-381 pairing checks for verifying KZG proofs: the reference's
 * check_proof_multi (FK20Py/kzg_proofs.py:207-232) pairs with py_ecc and has no
 * CUDA counterpart.  G2 points are on the twist y^2 = x^3 + 4(1 + u) over
 * Fp2 = Fp[u]/(u^2 + 1), an Fp2 element being {c0, c1} = c0 + c1 u; g2p_t is
 * homogeneous projective in standard form, infinity written as (0, 1, 0).
 * The pairing is the optimal ate pairing of BLS12 curves (up to a fixed
 * exponent: non-degenerate and bilinear, which is what the checks use).  One
 * thread per check; a launch takes about 34 ms whatever its count up to ~10^4
 * checks (B200; 280 k checks/s at 9,472). */
typedef struct { fp_t x[2], y[2], z[2]; } g2p_t;

/* ok[i] = (e(a[i], b[i]) == e(c[i], d[i])); a KZG multiproof check is
 * e(C - [I(s)]G1, G2) == e(proof, [s^l - x^l]G2). */
int fk20_pairing_check_n(uint8_t *ok, const g1p_t *a, const g2p_t *b, const g1p_t *c, const g2p_t *d, size_t count,
                         void *stream);
/* check_proof_multi (FK20Py/kzg_proofs.py:207-232) for count proofs at once:
 * ok[i] = 1 when proof[i] proves f(x[i] w^k) = ys[l i + k] for k < l (w = the
 * l-th root of unity 5^((r-1)/l), l a power of two <= 32) for the polynomial
 * committed in commitment[i]; else 0.  The G1 half of the setup comes from
 * the context's commitment tables (fk20_ctx_load_commit, n >= 32);
 * setup_g2 holds [s^k]G2 for k = 0..l (device memory, as the reference's
 * setup[1]).  The check is e(C - [I(s)]G1 + [x^l] proof, G2) ==
 * e(proof, [s^l]G2), I the interpolation polynomial of ys over the coset:
 * the reference's equation with x^l moved from G2 to G1.  All pointers are
 * device memory; count <= 2^20. */
int fk20_ctx_check_proof_multi(fk20_ctx *ctx, uint8_t *ok, const g1p_t *commitment, const g1p_t *proof,
                               const fr_t *x, const fr_t *ys, unsigned l, const g2p_t *setup_g2, unsigned count,
                               void *stream);
/* out[i][12] = e(a[i], b[i]) as the 6 Fp2 coefficients of w in Fp12 = Fp2[w]/(w^6 - (1 + u)): the
 * Miller value over |z| with the final exponent 3 (p^12 - 1)/r */
int fk20_pairing_n(fp_t *out, const g1p_t *a, const g2p_t *b, size_t count, void *stream);
/* G2 element-wise: 0 add, 1 dbl, 2 neg, 3 sub, 4 mul by fr_t scalar (b), 5 normalise,
 * 6 on-curve flag (b: uint8 out). */
int g2p_op_n(int op, g2p_t *out, const g2p_t *a, const void *b, size_t count, void *stream);

/* ------------------------------------------------------------------ request server
 * Continuous batching of blob-proof requests (no reference counterpart: the
 * reference has no serving layer).  A worker thread admits requests as they
 * arrive: whenever one of `slots` slots (a stream, a workspace, device and
 * pinned staging buffers) is free, it packs the waiting requests -- mixed
 * lengths, oldest first, up to max_rows and the device-memory budget -- and
 * enqueues them as one segment pipeline (one MSM launch and one persistent
 * G1 FFT launch over all lengths).  While few requests wait (latency mode)
 * a pack takes them all and its FFT may fill the GPU; when more wait
 * (throughput mode) a pack keeps whole groups of 32 rows per length and
 * packs of different slots split the SMs and run side by side.  Requests
 * that arrive meanwhile wait for the next free slot.
 * Slot buffers are sized for a full pack at creation when that fits the
 * budget.  The setup tables stay resident in the context (load every
 * length the requests use first).  Each request's result is the same as a
 * fk20_ctx_poly2h_fft of that polynomial alone.
 */
typedef struct fk20_server fk20_server;
typedef struct {
    unsigned max_rows;  /* requests per pack (1..4096; 0 = 160) */
    unsigned slots;     /* packs in flight at once (1..8; 0 = 2) */
    size_t hbm_budget;  /* device bytes all slots' buffers may hold (0 = half the free memory at creation);
                           a pack is also admitted only while what it adds to its slot's buffers is free
                           on the device when it is formed (less a 256 MiB reserve) */
    unsigned max_queue; /* waiting requests beyond which submit returns FK20_EAGAIN (0 = 1 << 16) */
    unsigned fft_blocks_per_sm; /* persistent-FFT blocks per SM of each pack.  0 = adaptive: the kernel's
                                   occupancy in latency mode (a pack may fill the GPU, and the next one's blocks
                                   take over as its blocks retire), occupancy / slots in throughput mode (packs
                                   split the SMs and run side by side) */
    unsigned latency_rows;      /* latency mode while at most this many requests wait: a pack takes them all;
                                   beyond it, throughput mode: packs of up to max_rows, whole 32-row groups per
                                   length (0 = max_rows; <= max_rows) */
    unsigned burst_rows;        /* pack size while more than 2 max_rows requests wait: larger packs drain a
                                   backlog faster (0 = 7/5 max_rows, i.e. 224 for 160; max_rows..4096) */
    unsigned engine;            /* 0: packs on slots (above).  1: cohorts -- continuous batching at FFT-stage
                                   granularity: the waiting requests of one length form a cohort as soon as a
                                   32-row group is full or the oldest has waited form_ms; its toeplitz + MSM
                                   run on their own stream, and every persistent-FFT launch advances all
                                   cohorts in flight by stages_per_launch stages, so a new cohort joins the
                                   next launch instead of waiting for a slot.  max_rows, slots, latency_rows,
                                   burst_rows and fft_blocks_per_sm apply to engine 0 only. */
    unsigned cohort_rows;       /* engine 1: rows per cohort at most (32..256; 0 = 64) */
    unsigned cohorts;           /* engine 1: cohorts in flight at most (1..24; 0 = 16) */
    unsigned form_ms;           /* engine 1: longest wait before a partial 32-row group is proved (0 = 25) */
    unsigned stages_per_launch; /* engine 1: FFT stages per persistent launch (1..17; 0 = 3) */
} fk20_server_config;
typedef struct {
    uint64_t requests, proofs, packs;
    double p50_ms, p99_ms, mean_ms, max_ms; /* latency: submit -> proofs in the caller's buffer */
    double wall_s;                          /* first submit -> last completion since the last reset */
    double proofs_per_s;                    /* proofs / wall_s */
    double mean_pack_rows;
    uint64_t rejected; /* submits refused with FK20_EAGAIN (max_queue requests waiting) */
    uint64_t nomem;    /* requests failed with FK20_ENOMEM (too large for the device memory alone) */
    uint64_t cancelled; /* requests cancelled with fk20_server_cancel before they were packed */
    double mean_wait_ms;    /* submit -> the request's pack is formed (mean over requests) */
    double mean_enqueue_ms; /* host time to stage and enqueue a pack (mean over packs) */
    double mean_run_ms;     /* pack enqueued -> its proofs copied out (mean over packs) */
    double mean_msm_ms;     /* engine 1: cohort staged -> the iteration with its MSM enqueued (mean over cohorts) */
    double mean_launch_ms;  /* engine 1: one FFT launch, enqueued -> done (mean over launches) */
    uint64_t launches;      /* engine 1: FFT launches */
} fk20_server_stats;
int fk20_server_create(fk20_server **srv, fk20_ctx *ctx, const fk20_server_config *cfg);
/* poly: HOST array of n fr_t (n in 1024, 2048, 4096); h_fft: HOST array of
 * 2n/16 g1p_t.  Both must stay valid until fk20_server_wait reports the
 * ticket done. */
int fk20_server_submit(fk20_server *srv, const fr_t *poly, unsigned n, g1p_t *h_fft, uint64_t *ticket);
/* 0: done, result written (the ticket is then forgotten); FK20_EAGAIN: not
 * done within timeout_ms (< 0 waits without limit); else the error of its pack. */
int fk20_server_wait(fk20_server *srv, uint64_t ticket, int timeout_ms);
/* Cancels a request that is still waiting for a pack: 0 (its buffers are
 * free again at once; fk20_server_wait then reports FK20_ECANCELED);
 * FK20_EAGAIN when it is already in a pack on the GPU (it completes
 * normally); FK20_EINVAL for an unknown or finished ticket. */
int fk20_server_cancel(fk20_server *srv, uint64_t ticket);
int fk20_server_get_stats(fk20_server *srv, fk20_server_stats *stats);
int fk20_server_reset_stats(fk20_server *srv);
/* Finishes every submitted request, then stops the worker and frees the slots. */
int fk20_server_destroy(fk20_server *srv);

/* ------------------------------------------------------------------ reference entry points
 * These use a process-wide default context on the current device; tables are
 * rebuilt when the content of xext_fft changes (checked by a device-side
 * fingerprint).  n = 4096, m = 512, rows <= 2^20.
 */

/* fk20_poly2h_fft.cu:47 -- polynomial[rows][4096] + xext_fft[16][512] -> h_fft[rows][512] */
int fk20_poly2h_fft(g1p_t *h_fft, const fr_t *polynomial, const g1p_t *xext_fft, unsigned rows);

/* No counterpart in the reference (whose tables live in file-scope managed
 * memory for the life of the process): frees the default context of `device`
 * and its tables (117 GB at window 15); the next reference-signature call on
 * that device builds them again.  No call may be in flight on it. */
int fk20_default_release(int device);

/* No counterpart in the reference (it has no checked build; its debug build
 * asserts).  In the checked build (libfk20b200_checked.so, `make checked`)
 * the MSM and the persistent G1 FFT check their task decoding, tile and table
 * indices and the signed-digit recoding against the sizes they were given;
 * a failure is recorded, never trapped, and the access skipped.  Waits for
 * the device, then returns the first failing site since the last call
 * (FK20_CHECK_* below; 0: none) and clears it; *compiled (if not null) is 1
 * in the checked build, 0 in the normal one, where nothing is checked. */
#define FK20_CHECK_MSM_TILE 1     /* MSM: warp outside its segment's tiles */
#define FK20_CHECK_MSM_CARRY 2    /* MSM: a scalar needs more windows than its table has */
#define FK20_CHECK_MSM_PLANTED 3  /* MSM: the test hook FK20_OPT_TEST_CHECK */
#define FK20_CHECK_FFT_TASK 11    /* persistent FFT: task decoded outside its segment */
#define FK20_CHECK_FFT_PROGRAM 12 /* persistent FFT: twiddle program index out of range */
int fk20_check_status(int *compiled);

/* No counterpart in the reference.  For tests of the out-of-memory paths
 * only: the next `count` device allocations the library makes fail as if
 * the device were full (FK20_ENOMEM); 0 ends the injection. */
int fk20_test_fail_allocations(int count);

/* fk20_poly2toeplitz_coefficients.cu:25 -- polynomial[rows][4096] -> tc[rows][16][512] */
int fk20_poly2toeplitz_coefficients(fr_t *toeplitz_coefficients, const fr_t *polynomial, unsigned rows,
                                    void *stream);

/* fk20_poly2toeplitz_coefficients_fft.cu:24 -- polynomial -> tc_fft[rows][16][512] */
int fk20_poly2toeplitz_coefficients_fft(fr_t *toeplitz_coefficients_fft, const fr_t *polynomial, unsigned rows,
                                        void *stream);

/* fk20_poly2hext_fft.cu:26 -- polynomial + xext_fft -> hext_fft[rows][512] */
int fk20_poly2hext_fft(g1p_t *hext_fft, const fr_t *polynomial, const g1p_t *xext_fft, unsigned rows, void *stream);

/* fk20_msm.cu:23 -- tc_fft[rows][16][512] + xext_fft[16][512] -> hext_fft[rows][512] */
int fk20_msm(g1p_t *hext_fft, const fr_t *toeplitz_coefficients_fft, const g1p_t *xext_fft, unsigned rows,
             void *stream);

/* fk20_hext_fft2h_fft.cu:27 -- hext_fft[rows][512] -> h_fft[rows][512]
 * (inverse FFT, upper half set to infinity, forward FFT) */
int fk20_hext_fft2h_fft(g1p_t *h_fft, const g1p_t *hext_fft, unsigned rows, void *stream);

/* fk20.cuh:24 -- hext_fft -> h (inverse FFT, upper half infinity) */
int fk20_hext_fft2h(g1p_t *h, const g1p_t *hext_fft, unsigned rows, void *stream);

/* fk20.cu:74 -- hext_fft -> hext (inverse FFT) */
int fk20_hext_fft2hext(g1p_t *hext, const g1p_t *hext_fft, unsigned rows, void *stream);

/* fk20.cu:94 -- h -> h_fft (forward FFT) */
int fk20_h2h_fft(g1p_t *h_fft, const g1p_t *h, unsigned rows, void *stream);

/* fk20_poly2h_fft.cu:27 -- h[rows][512]: entries 256..511 set to infinity, in place */
int fk20_hext2h(g1p_t *h, unsigned rows, void *stream);

/* fk20.cu:28 -- setup[>= 4080] -> xext_fft[16][512] */
int fk20_setup2xext_fft(g1p_t *xext_fft, const g1p_t *setup, void *stream);

/* fr_fft.cu:318 / :347 (fr_fft_wrapper, fr_ift_wrapper) -- `count` independent
 * 512-point transforms over Fr, natural order in and out; the inverse includes
 * the 1/512 factor.  Input and output may alias. */
int fr_fft(fr_t *output, const fr_t *input, unsigned count, void *stream);
int fr_ift(fr_t *output, const fr_t *input, unsigned count, void *stream);

/* g1p_fft.cu:337 / :350 (g1p_fft_wrapper, g1p_ift_wrapper) -- `count`
 * independent 512-point transforms over G1, natural order; the inverse
 * includes the 1/512 factor.  Input and output may alias. */
int g1p_fft(g1p_t *output, const g1p_t *input, unsigned count, void *stream);
int g1p_ift(g1p_t *output, const g1p_t *input, unsigned count, void *stream);

/* Size-generic transforms: log_m in 1..9. */
int fr_fft_n(fr_t *output, const fr_t *input, unsigned log_m, unsigned count, int inverse, void *stream);
int g1p_fft_n(g1p_t *output, const g1p_t *input, unsigned log_m, unsigned count, int inverse, void *stream);

/* No counterpart in the reference.  The same transforms as g1p_fft_n for
 * callers that must not have the library allocate device memory (their
 * memory is owned by their own allocator or pool, or they cannot take the
 * device-wide synchronisation of cudaMalloc/cudaFree): the working tiles live
 * in a fixed file-scope device array of ~4.7 MB that every GPU loading the
 * library holds until exit.  At most 64 transforms (log_m <= 9) per call;
 * more returns FK20_ETOOBIG.  The first call on a device looks up the array's
 * address (under lazy module loading, that is also when the array's memory is
 * committed): make it at start-up, before any stream capture.  The address
 * is cached per device for the life of the process: do not reset a device
 * (cudaDeviceReset) while this entry point is in use.  All calls share the
 * array: calls that overlap on the GPU race and must be serialised. */
int g1p_fft_noalloc(g1p_t *output, const g1p_t *input, unsigned log_m, unsigned count, int inverse, void *stream);

/* ------------------------------------------------------------------ element-wise helpers
 * Batched forms of the fp_* / fr_* / g1p_* device API (fp.cuh:16-41,
 * fr.cuh:33-58, g1.cuh:31-96), for tests, microbenchmarks and callers that
 * need single operations.  op codes:
 *   field: 0 mul, 1 sqr, 2 add, 3 sub, 4 neg, 5 inv, 6 reduce (canonical),
 *          7 x2, 8 x3, 9 x4, 10 x8, 11 x12
 *   g1p:   0 add, 1 dbl, 2 neg, 3 sub, 4 mul by fr_t scalar, 5 normalise
 *          (affine {x, y, 1}, infinity (0, 1, 0)), 6 is_point (b: uint8 out)
 */
int fp_op_n(int op, fp_t *out, const fp_t *a, const fp_t *b, size_t count, void *stream);
int fr_op_n(int op, fr_t *out, const fr_t *a, const fr_t *b, size_t count, void *stream);
int g1p_op_n(int op, g1p_t *out, const g1p_t *a, const void *b, size_t count, void *stream);

/* fr.cu:99 / g1p.cu:142 -- eq[i] = (x[i] == y[i]) mathematically */
int fr_eq_n(uint8_t *eq, const fr_t *x, const fr_t *y, size_t count, void *stream);
int g1p_eq_n(uint8_t *eq, const g1p_t *p, const g1p_t *q, size_t count, void *stream);

/* g1p.cu:168 -- affine conversion of count points (infinity -> (0, 0)) */
int g1a_fromG1p_n(g1a_t *a, const g1p_t *p, size_t count, void *stream);

/* Microbenchmark of the Montgomery product: `iters` dependent products per
 * element on `count` elements of limb-major Montgomery data (field 0 = Fp,
 * 1 = Fr; sqr != 0 squares).  data: count x N 32-bit words, limb-major
 * (word k of element e at data[k * count + e]). */
int fk20_bench_field(int field, int sqr, uint32_t *data, size_t count, int iters, void *stream);

/* IMAD-pipe peak probe: blocks x threads threads, each running iters x 32
 * independent 32-bit multiply-adds (8 chains); the caller times it.  The
 * roofline denominator for this integer workload. */
int fk20_bench_imad(uint32_t *sink, int blocks, int threads, int iters, void *stream);

/* Engine version string. */
const char *fk20_version(void);

#ifdef __cplusplus
}
#endif

#endif /* FK20_B200_H */
