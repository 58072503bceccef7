// engine.cu -- host side of the B200 FK20 engine and its C ABI (include/fk20_b200.h).
//
// Owns
//   - the constant tables (GLV/wNAF twiddle programs, Fr twiddles), computed
//     once on the host from the curve constants and uploaded to every kernel
//     module of every device used;
//   - contexts: fixed-base MSM tables per polynomial length, commitment
//     tables, options, a workspace;
//   - the segment pipeline (run_segments): toeplitz Fr FFTs, one MSM launch
//     and one persistent G1 FFT launch over up to 8 segments, outputs;
//   - batch plans (CUDA graphs of that pipeline), the autotuner, and the
//     continuous-batching request server (a worker thread and its slots);
//   - the launch sequence of every entry point.
// There is no CPU compute path: without a usable sm_100 device every entry
// point returns FK20_ENODEV or the CUDA error.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "../../include/fk20_b200.h"
#include "check.cuh"
#include "consts.cuh"
#include "launch.h"
#include "layout.cuh"

using namespace fk;

#define FK20_VERSION "fk20-b200 0.1 (sm_100a)"

namespace fk {

static void fr_std_to_u64(uint64_t out[4], const Fr &s) {
    for (int k = 0; k < 4; k++) out[k] = (uint64_t)s.w[2 * k] | ((uint64_t)s.w[2 * k + 1] << 32);
}

// Twiddle programs and Fr constants, computed with the host build of the
// field code: w_512 = 5^((r-1)/512) (FK20Py/kzg_proofs.py:39-44), its powers
// (the reference's fr_roots table, fr_roots.cu:17-533) and 2^-s.
const HostConsts &host_consts() {
    static HostConsts hc;
    static std::once_flag once;
    std::call_once(once, [] {
        Fr five, w, acc, t;
        f_set_zero(t);
        t.w[0] = 5;
        f_to_mont(five, t);
        uint32_t e[8];
        for (int i = 0; i < 8; i++) e[i] = FrDesc::mod(i);
        e[0] -= 1;  // r - 1 (the low word of r is 1)
        for (int i = 0; i < 8; i++) e[i] = (e[i] >> 9) | (i < 7 ? (e[i + 1] << 23) : 0);  // (r-1)/512
        f_pow(w, five, e, 8);
        f_set_one(acc);
        for (int k = 0; k < 512; k++) {
            for (int i = 0; i < 8; i++) hc.fr_tw[k][i] = acc.w[i];
            Fr s;
            f_from_mont(s, acc);
            uint64_t k64[4];
            fr_std_to_u64(k64, s);
            host::make_program(hc.prog[k], k64);
            f_mul(acc, acc, w);
        }
        Fr half, two, p2;
        f_set_zero(t);
        t.w[0] = 2;
        f_to_mont(two, t);
        f_inv(half, two);
        f_set_one(p2);
        for (int s = 0; s < 16; s++) {
            for (int i = 0; i < 8; i++) hc.fr_inv2[s][i] = p2.w[i];
            Fr st;
            f_from_mont(st, p2);
            uint64_t k64[4];
            fr_std_to_u64(k64, st);
            host::make_program(hc.prog[512 + s], k64);
            f_mul(p2, p2, half);
        }
        for (int k = 0; k < NPROG; k++) host::program_cost(hc.prog[k], &hc.prog_dbl[k], &hc.prog_add[k]);
    });
    return hc;
}

}  // namespace fk

namespace {

std::mutex g_dev_mu;
bool g_dev_ready[64];

int ensure_device(int dev) {
    if (dev < 0 || dev >= 64) return FK20_ENODEV;
    std::lock_guard<std::mutex> lk(g_dev_mu);
    if (g_dev_ready[dev]) return 0;
    cudaDeviceProp prop;
    cudaError_t err = cudaGetDeviceProperties(&prop, dev);
    if (err != cudaSuccess) { cudaGetLastError(); return FK20_ENODEV; }
    if (prop.major < 10) return FK20_ENODEV;
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != dev) cudaSetDevice(dev);
    err = upload_consts_fr();
    if (err == cudaSuccess) err = upload_consts_msm();
    if (err == cudaSuccess) err = upload_consts_fft();
    if (err == cudaSuccess) err = upload_consts_tables();
    if (err == cudaSuccess) err = upload_consts_misc();
    if (cur != dev) cudaSetDevice(cur);
    if (err != cudaSuccess) return (int)err;
    g_dev_ready[dev] = true;
    return 0;
}

int current_device_ready() {
    int dev;
    if (cudaGetDevice(&dev) != cudaSuccess) { cudaGetLastError(); return FK20_ENODEV; }
    return ensure_device(dev);
}

}  // namespace

namespace fk {
// constant tables uploaded to the current device (used by noalloc.cu)
int device_ready() { return current_device_ready(); }
}  // namespace fk

namespace {

#define CK(x)                                  \
    do {                                       \
        cudaError_t e_ = (x);                  \
        if (e_ != cudaSuccess) return (int)e_; \
    } while (0)
#define CKL()                                  \
    do {                                       \
        cudaError_t e_ = cudaGetLastError();   \
        if (e_ != cudaSuccess) return (int)e_; \
    } while (0)
#define CKR(x)                   \
    do {                         \
        int r_ = (x);            \
        if (r_ != 0) return r_;  \
    } while (0)

inline cudaStream_t S_(void *s) { return (cudaStream_t)s; }

// n -> log_m (m = 2n/16) for the supported lengths
int log_m_for_n(unsigned n) {
    switch (n) {
    case 1024: return 7;
    case 2048: return 8;
    case 4096: return 9;
    default: return -1;
    }
}

constexpr unsigned MAX_ROWS = 1u << 20;
// The FK20 MSM's tables cover the 128-bit GLV halves of the scalars (glv.cuh;
// signed digits need one bit more); windows 8..15.
constexpr int GLV_TABLE_BITS = 129;
constexpr int MAX_WINDOW = 15;

// the persistent FFT's error word: 1000 + stage when a bounded wait gave up,
// 2000 when a check of the checked build stopped the launch
int launch_error(int e) { return e >= 2000 ? FK20_ECHECK : FK20_ETIMEOUT; }

// A device buffer that only grows.  The buffer it outgrows may still be read
// by work queued on any stream, and cudaFree would wait for the whole device
// (stalling, for instance, a server's other packs): it is kept until
// release() instead, when the owner is torn down.  Growth is geometric in
// practice (a larger batch, a longer polynomial), so the kept buffers hold
// less than the live one.
// fk20_test_fail_allocations: device allocations still to fail (tests of the
// out-of-memory paths)
std::atomic<int> g_fail_allocs{0};
bool injected_alloc_failure() {
    int left = g_fail_allocs.load();
    while (left > 0 && !g_fail_allocs.compare_exchange_weak(left, left - 1)) {
    }
    return left > 0;
}

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    std::vector<void *> outgrown;
    int reserve(size_t need) {
        if (need <= bytes) return 0;
        if (injected_alloc_failure()) return FK20_ENOMEM;
        void *q = nullptr;
        if (cudaMalloc(&q, need) != cudaSuccess) {
            cudaGetLastError();
            return FK20_ENOMEM;
        }
        if (p) outgrown.push_back(p);
        p = q;
        bytes = need;
        return 0;
    }
    void release() {
        for (void *q : outgrown) cudaFree(q);
        outgrown.clear();
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
};

struct Tables {
    bool ready = false;
    unsigned n = 0;
    int log_m = 0, cb = 0, W = 0;
    DevBuf table;
    DevBuf xext;             // the xext_fft the tables were built from (rebuilds at another window)
    unsigned gen = 0;        // bumped at every build: graph plans check it before replaying
    unsigned long long fingerprint = 0;
};

// Device state of one in-flight pipeline call: scalar and point tiles, the
// offset arrays of ragged batches, and the persistent launch's counters.  A
// context owns one; every batch plan and server slot owns its own, so that
// they can run on different streams at once against the same tables.
struct Workspace {
    DevBuf S, D, offs, sync;           // sync: [task counter | error flag | pad][readiness counters]
    int *err_host = nullptr;           // pinned copy of the last persistent launch's error flag
    size_t *offs_host = nullptr;       // pinned staging of offset arrays
    size_t offs_cap = 0;               // entries of offs_host
    cudaEvent_t offs_done = nullptr;   // the last copy out of offs_host
    int init() {
        if (err_host) return 0;
        if (cudaMallocHost(&err_host, sizeof(int)) != cudaSuccess) {
            cudaGetLastError();
            err_host = nullptr;
            return FK20_ENOMEM;
        }
        *err_host = 0;
        return 0;
    }
    // pinned staging for `count` offsets with no copy out of it pending
    int stage_offsets(size_t count) {
        if (offs_done) {
            CK(cudaEventSynchronize(offs_done));
        } else {
            CK(cudaEventCreateWithFlags(&offs_done, cudaEventDisableTiming));
        }
        if (count > offs_cap) {
            if (offs_host) cudaFreeHost(offs_host);
            offs_host = nullptr;
            offs_cap = 0;
            if (cudaMallocHost(&offs_host, count * sizeof(size_t)) != cudaSuccess) {
                cudaGetLastError();
                return FK20_ENOMEM;
            }
            offs_cap = count;
        }
        return 0;
    }
    size_t bytes() const { return S.bytes + D.bytes + offs.bytes + sync.bytes; }
    void release() {
        S.release();
        D.release();
        offs.release();
        sync.release();
        if (err_host) cudaFreeHost(err_host);
        if (offs_host) cudaFreeHost(offs_host);
        if (offs_done) cudaEventDestroy(offs_done);
        err_host = nullptr;
        offs_host = nullptr;
        offs_cap = 0;
        offs_done = nullptr;
    }
};

}  // namespace

// Per-launch profiling: CUDA events on the launching stream around every
// pipeline kernel, with the algorithmic work of that launch (in 32x32->64-bit
// limb products: Fp product M_p = 300, Fr product M_r = 136, RCB addition
// 12 M_p, XYZZ mixed addition 10 M_p, doubling 8 M_p).
// NVTX ranges per pipeline stage (toeplitz + Fr FFTs, MSM, G1 FFT stages,
// output), named "fk20 <stage>", for nsys / ncu timelines: on when the
// environment variable FK20_NVTX is set to a nonzero value (read once per
// process).  Ranges are started and ended by id, so an error return between
// a stage's launch and its end leaves no nesting unbalanced.
bool nvtx_on() {
    static const bool on = [] {
        const char *e = getenv("FK20_NVTX");
        return e && atoi(e) != 0;
    }();
    return on;
}
const char *const NVTX_STAGE[FK20_NKINDS] = {"fk20 tc_fft", "fk20 msm",    "fk20 stage_inv", "fk20 stage_fwd",
                                             "fk20 middle", "fk20 output", "fk20 fft_fused"};

struct Profiler {
    bool on = false;
    nvtxRangeId_t nvtx = 0;
    struct Rec {
        int kind;
        double products, executed;
        cudaEvent_t a, b;
    };
    std::vector<Rec> pending;
    std::vector<cudaEvent_t> pool;
    double ms[FK20_NKINDS] = {0}, products[FK20_NKINDS] = {0}, executed[FK20_NKINDS] = {0};
    long launches[FK20_NKINDS] = {0};
    cudaEvent_t get() {
        if (!pool.empty()) {
            cudaEvent_t e = pool.back();
            pool.pop_back();
            return e;
        }
        cudaEvent_t e;
        cudaEventCreate(&e);
        return e;
    }
    // `alg` algorithmic and `exe` executed limb products of the launch
    void begin(int kind, double alg, double exe, cudaStream_t st) {
        if (nvtx_on()) nvtx = nvtxRangeStartA(NVTX_STAGE[kind]);
        if (!on) return;
        Rec r{kind, alg, exe, get(), get()};
        cudaEventRecord(r.a, st);
        pending.push_back(r);
    }
    void end(cudaStream_t st) {
        if (nvtx) {
            nvtxRangeEnd(nvtx);
            nvtx = 0;
        }
        if (!on || pending.empty()) return;
        cudaEventRecord(pending.back().b, st);
    }
    void collect() {
        for (Rec &r : pending) {
            cudaEventSynchronize(r.b);
            float t = 0;
            cudaEventElapsedTime(&t, r.a, r.b);
            ms[r.kind] += t;
            products[r.kind] += r.products;
            executed[r.kind] += r.executed;
            launches[r.kind] += 1;
            pool.push_back(r.a);
            pool.push_back(r.b);
        }
        pending.clear();
    }
    void reset() {
        collect();
        for (int k = 0; k < FK20_NKINDS; k++) ms[k] = products[k] = executed[k] = 0, launches[k] = 0;
    }
    ~Profiler() {
        for (Rec &r : pending) pool.push_back(r.a), pool.push_back(r.b);
        for (cudaEvent_t e : pool) cudaEventDestroy(e);
    }
};

struct fk20_ctx {
    int device = 0;
    int window = 10;
    int sms = 148;
    int fused_fft = 1;          // run the G1 FFT stages as one persistent launch
    int msm_threads = 128;      // MSM block size (64, 128, 256)
    int test_check = 0;         // checked build: MSM launches record a planted failure (tests)
    int fft_blocks_per_sm = 0;  // persistent FFT grid: blocks per SM (0 = as many as fit)
    int fused_occupancy = 1;    // blocks of the persistent FFT kernel that fit on one SM
    unsigned wait_limit = FUSED_SPIN_LIMIT;  // polls before a persistent wait gives up
    unsigned unpublished = 0xffffffffu;      // test hook: a task whose completion is not published
    std::mutex mu;
    Tables tab[3];  // log_m 7, 8, 9
    struct {        // KZG commitment tables over setup points s_0 .. s_{n-1}
        DevBuf table, part;
        int n = 0, cb = 0, W = 0;
    } commit;
    Workspace ws;   // the context's own calls
    DevBuf D2, scratch, xext, fp_dev;
    DevBuf verify;  // check_proof_multi intermediates
    Profiler prof;
};

namespace {

Tables *tables_for(fk20_ctx *ctx, int log_m) { return (log_m >= 7 && log_m <= 9) ? &ctx->tab[log_m - 7] : nullptr; }

size_t tile_bytes(int G, int m) { return (size_t)G * m * TILE_Q * 32 * sizeof(uint4); }
size_t scal_bytes(int G, int m) { return (size_t)G * m * L_COLS * SCAL_Q * 32 * sizeof(uint4); }

struct DeviceGuard {  // make ctx->device current for the duration of a call
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev); else prev = -1;
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

// ---- work model (limb products) -----------------------------------------------
// Two accountings of each launch, both in 32x32->64-bit limb products.
//
// Algorithmic (`alg`): the fixed unit costs of the FK20 work, independent of
// the formulas a kernel uses -- an Fp product or square 300 limb products
// (12-limb CIOS: 2 x 12^2 + 12), an Fr product 136; a G1 addition 12, mixed
// addition 11 and doubling 8 Fp products (the complete projective formulas
// of Renes-Costello-Batina, a = 0); a fixed-scalar multiplication costs its
// chain's doublings and additions at those prices.  This is the work that
// the roofline fraction divides by.
//
// Executed (`exe`): the products the kernels actually run with their cheaper
// formulas -- a triangular square 234 (78 + 156), the MSM's mixed addition
// into an XYZZ accumulator 8 M + 2 S, the twiddle programs' Jacobian
// doublings and mixed additions on the isomorphic curve (below).
constexpr double MP = 300.0, MR = 136.0, ADD_P = 12 * MP;
constexpr double MADD_A = 11 * MP, DBL_A = 8 * MP;
constexpr double MS_X = 234.0, MADD_X = 8 * MP + 2 * MS_X, DBL_X = 6 * MP + 2 * MS_X;

struct Work {
    double alg = 0, exe = 0;
    Work() = default;
    Work(double a, double e) : alg(a), exe(e) {}
    explicit Work(double both) : alg(both), exe(both) {}
    Work &operator+=(const Work &o) { alg += o.alg, exe += o.exe; return *this; }
    Work operator*(double k) const { return Work(alg * k, exe * k); }
    Work operator+(const Work &o) const { return Work(alg + o.alg, exe + o.exe); }
};

// A twiddle program (scalar_prog.cuh).  Algorithmic: its chain's doublings
// and additions (program_cost counts the 3P, 5P, 7P precompute's doubling and
// three additions with the digits') plus phi(P).  Executed: P to Jacobian
// (2 M + 1 S), 2P with P on its Z (2 M + 5 S), 3P, 5P, 7P by co-Z additions
// (3 x (5 M + 2 S)), the points brought onto one Z (11 M + 3 S) with their
// phi images (4 M), the result brought back (3 M + 1 S): 37 M + 16 S; then
// Jacobian doublings (2 M + 5 S) and mixed additions (8 M + 3 S).
Work prog_products(int idx) {
    const HostConsts &hc = host_consts();
    if (hc.prog[idx][0] & 0x300u) return Work();
    const double dbl = hc.prog_dbl[idx], add = hc.prog_add[idx];
    return Work(dbl * DBL_A + add * ADD_P + MP,
                37.0 * MP + 16.0 * MS_X + (dbl - 1) * (2 * MP + 5 * MS_X) + (add - 3) * (8 * MP + 3 * MS_X));
}

// one stage over `rows` rows: kind 0 DIF inverse, 1 DIT forward
Work stage_products(int rows, int log_m, int s, int kind) {
    const int m = 1 << log_m;
    Work per_row;
    for (int b = 0; b < m / 2; b++) {
        int tix;
        if (kind == 0) {
            const int half = m >> (s + 1), j = b & (half - 1);
            tix = ((m - (j << s)) << (MAX_LOG_M - log_m)) & 511;
        } else {
            const int half = 1 << s, j = b & (half - 1);
            tix = (j << (log_m - 1 - s)) << (MAX_LOG_M - log_m);
        }
        per_row += Work(2 * ADD_P) + (tix ? prog_products(tix) : Work());
    }
    return per_row * rows;
}

Work fr_fft_products(int log_m) {  // nontrivial twiddle products of one Fr FFT-m
    const int m = 1 << log_m;
    return Work(((double)log_m * (m / 2) - (m - 1)) * MR);
}

// the fixed-base MSM per output point: 16 terms x 2W window additions (W
// windows on each GLV half), phi once, and (times_m) log_m doublings
Work msm_products(int W, int log_m, bool times_m) {
    Work w(L_COLS * 2 * W * MADD_A + MP, L_COLS * 2 * W * MADD_X + MP);
    if (times_m) w += Work(log_m * DBL_A, log_m * DBL_X);
    return w;
}

// inverse DIF stages 0..L-2, middle (last inverse + zero upper half + first
// forward stage, optionally times 1/m), forward DIT stages 1..L-1
int run_hext_to_hfft(Profiler &pf, uint4 *D, int G, int rows, int log_m, int scale, cudaStream_t st) {
    const int m = 1 << log_m;
    for (int s = 0; s < log_m - 1; s++) {
        const Work w = stage_products(rows, log_m, s, 0);
        pf.begin(FK20_K_STAGE_INV, w.alg, w.exe, st);
        launch_g1_stage(D, G, log_m, s, 0, st);
        pf.end(st);
        CKL();
    }
    const Work mid = (Work(ADD_P) + (scale ? prog_products(512 + log_m) : Work())) * ((double)rows * (m / 2));
    pf.begin(FK20_K_MIDDLE, mid.alg, mid.exe, st);
    launch_g1_middle(D, G, log_m, scale, st);
    pf.end(st);
    CKL();
    for (int s = 1; s < log_m; s++) {
        const Work w = stage_products(rows, log_m, s, 1);
        pf.begin(FK20_K_STAGE_FWD, w.alg, w.exe, st);
        launch_g1_stage(D, G, log_m, s, 1, st);
        pf.end(st);
        CKL();
    }
    return 0;
}

int output_launch(Profiler &pf, uint64_t *dst, const uint4 *D, const size_t *row_off, int rows, int log_m,
                  int bitrev_out, cudaStream_t st) {
    pf.begin(FK20_K_OUTPUT, (double)rows * (1 << log_m) * 3 * MP, (double)rows * (1 << log_m) * 3 * MP, st);
    launch_tile_to_ref(dst, D, row_off, rows, log_m, bitrev_out, st);
    pf.end(st);
    CKL();
    return 0;
}

// Fixed-base tables of `nbases` bases (reference g1p_t on the device) at
// window cb, every base first multiplied by program prog_scale (< 0: none),
// for scalars of `bits` bits (W = ceil(bits / cb) windows).
int build_base_tables(fk20_ctx *ctx, DevBuf &table, const uint64_t *bases, int nbases, int cb, int prog_scale,
                      int bits, cudaStream_t st) {
    const int W = (bits + cb - 1) / cb;
    const int E = 1 << (cb - 1);
    const size_t entries = (size_t)nbases * W * E;
    table.release();
    CKR(table.reserve(entries * 6 * sizeof(uint4)));
    // slabs of bases keep the Z scratch near 1 GiB
    const size_t per_base_z = (size_t)W * E * table_z_bytes();
    int slab = (int)std::max<size_t>(1, (1ull << 30) / per_base_z);
    slab = std::min(slab, nbases);
    CKR(ctx->scratch.reserve((size_t)slab * per_base_z + (size_t)slab * W * table_window_base_bytes()));
    void *zs = ctx->scratch.p;
    void *wb = (char *)ctx->scratch.p + (size_t)slab * per_base_z;
    for (int b0 = 0; b0 < nbases; b0 += slab) {
        const int nb = std::min(slab, nbases - b0);
        launch_table_windows(wb, bases, b0, nb, W, cb, prog_scale, st);
        CKL();
        launch_table_fill((uint4 *)table.p, zs, wb, b0, nb, W, cb, st);
        CKL();
        launch_table_affine((uint4 *)table.p, zs, b0, nb, W, cb, st);
        CKL();
    }
    return 0;
}

int build_tables(fk20_ctx *ctx, int log_m, const uint64_t *xext, cudaStream_t st) {
    Tables *T = tables_for(ctx, log_m);
    const int m = 1 << log_m;
    const int cb = ctx->window;
    const int W = (GLV_TABLE_BITS + cb - 1) / cb;
    T->ready = false;
    T->gen++;
    if (xext != (const uint64_t *)T->xext.p) {  // keep the bases for rebuilds at another window
        CKR(T->xext.reserve((size_t)L_COLS * m * sizeof(g1p_t)));
        CK(cudaMemcpyAsync(T->xext.p, xext, (size_t)L_COLS * m * sizeof(g1p_t), cudaMemcpyDeviceToDevice, st));
        xext = (const uint64_t *)T->xext.p;
    }
    // the inverse FFT's 1/m folded into the bases (program 512 + log m = 2^-log m)
    CKR(build_base_tables(ctx, T->table, xext, L_COLS * m, cb, 512 + log_m, GLV_TABLE_BITS, st));
    T->n = (unsigned)(m * L_COLS / 2);
    T->log_m = log_m;
    T->cb = cb;
    T->W = W;
    // complete before returning: later calls may come on other streams (server
    // slots, plans, non-blocking caller streams) that do not order after `st`
    CK(cudaStreamSynchronize(st));
    T->ready = true;
    return 0;
}

int fingerprint(fk20_ctx *ctx, const void *p, size_t words, unsigned long long *out, cudaStream_t st) {
    CKR(ctx->fp_dev.reserve(sizeof(unsigned long long)));
    CK(cudaMemsetAsync(ctx->fp_dev.p, 0, sizeof(unsigned long long), st));
    launch_fingerprint((unsigned long long *)ctx->fp_dev.p, (const uint64_t *)p, words, st);
    CKL();
    CK(cudaMemcpyAsync(out, ctx->fp_dev.p, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return 0;
}

int msm_launch(fk20_ctx *ctx, Tables *T, uint4 *D, const uint4 *S, int G, int rows, int times_m, cudaStream_t st) {
    MsmArgs a{};
    a.seg[0] = MsmSeg{D, S, (const uint4 *)T->table.p, G, T->log_m, rows, T->cb, T->W, 0};
    a.nseg = 1;
    a.times_m = times_m;
    a.test_check = ctx->test_check;
    a.warps = (unsigned)G << T->log_m;
    const Work w = msm_products(T->W, T->log_m, times_m != 0) * ((double)rows * (1 << T->log_m));
    ctx->prof.begin(FK20_K_MSM, w.alg, w.exe, st);
    launch_msm(a, ctx->msm_threads, st);
    ctx->prof.end(st);
    CKL();
    return 0;
}

// One segment of a pipeline call: `rows` polynomials of length n = 8m
// (m = 2^log_m); polynomial r starts at word 4 * poly_off[r] of the input and
// its outputs at word 18 * out_off[r] of the output (device arrays; null =
// contiguous rows).
struct Seg {
    int log_m;
    unsigned rows;
    const size_t *poly_off, *out_off;
};

constexpr size_t SYNC_HDR = 256;  // persistent-launch header: task counter at 0, error flag at 128
// Fp products per compressed proof: inversion by Fermat (381 squarings + 190
// products), two products to affine, two conversions out of Montgomery form
constexpr double PROOF_OUT_MP = 575.0;

struct SegLayout {
    size_t s_off[MAX_SEGS], d_off[MAX_SEGS], r_off[MAX_SEGS];
    size_t s_bytes = 0, d_bytes = 0, r_bytes = 0;
};

int segment_layout(fk20_ctx *ctx, const Seg *sg, int nseg, SegLayout &lay) {
    if (nseg < 1 || nseg > MAX_SEGS) return FK20_EINVAL;
    for (int k = 0; k < nseg; k++) {
        Tables *T = tables_for(ctx, sg[k].log_m);
        if (!T) return FK20_EINVAL;
        if (!T->ready) return FK20_ENOSETUP;
        const int m = 1 << sg[k].log_m, G = (int)((sg[k].rows + 31) / 32);
        lay.s_off[k] = lay.s_bytes;
        lay.s_bytes += scal_bytes(G, m);
        lay.d_off[k] = lay.d_bytes;
        lay.d_bytes += tile_bytes(G, m);
        lay.r_off[k] = lay.r_bytes;
        lay.r_bytes += (size_t)G * m * sizeof(unsigned);
    }
    return 0;
}

// device buffers of a segment call (a no-op once they are large enough)
int reserve_segments(fk20_ctx *ctx, Workspace &ws, const Seg *sg, int nseg, bool full) {
    SegLayout lay;
    CKR(segment_layout(ctx, sg, nseg, lay));
    CKR(ws.init());
    CKR(ws.S.reserve(lay.s_bytes));
    CKR(ws.D.reserve(lay.d_bytes));
    if (full) CKR(ws.sync.reserve(SYNC_HDR + lay.r_bytes));
    return 0;
}

// Enqueues the FK20 pipeline of the segments on st: the toeplitz Fr FFTs (one
// launch per segment), ONE fixed-base MSM launch over all segments, then
// (full) the G1 inverse + forward transforms as ONE persistent launch over all
// segments -- or stage by stage when the fused FFT is off -- and the h_fft
// outputs; or (!full) the hext_fft outputs times m.  The tables are the
// context's; the workspace is the caller's.  Allocates only when `ws` is too
// small (reserve_segments first makes the enqueue allocation-free).
int run_segments(fk20_ctx *ctx, Workspace &ws, const Seg *sg, int nseg, const fr_t *polys, void *out, bool full,
                 cudaStream_t st, bool proofs = false, int fft_bps = 0) {
    SegLayout lay;
    CKR(segment_layout(ctx, sg, nseg, lay));
    CKR(reserve_segments(ctx, ws, sg, nseg, full));
    if (*ws.err_host) return launch_error(*ws.err_host);  // a previous persistent launch stopped: results invalid
    uint4 *S = (uint4 *)ws.S.p, *D = (uint4 *)ws.D.p;
    const size_t U = sizeof(uint4);
    for (int k = 0; k < nseg; k++) {
        Tables *T = tables_for(ctx, sg[k].log_m);
        const Work w = fr_fft_products(sg[k].log_m) * ((double)sg[k].rows * L_COLS);
        ctx->prof.begin(FK20_K_TC_FFT, w.alg, w.exe, st);
        launch_tc_fft(S + lay.s_off[k] / U, (const uint64_t *)polys, sg[k].poly_off, (int)T->n, sg[k].log_m,
                      sg[k].rows, st);
        ctx->prof.end(st);
        CKL();
    }
    MsmArgs a{};
    Work prod;
    unsigned warps = 0;
    for (int k = 0; k < nseg; k++) {
        Tables *T = tables_for(ctx, sg[k].log_m);
        const int m = 1 << sg[k].log_m, G = (int)((sg[k].rows + 31) / 32);
        a.seg[k] = MsmSeg{D + lay.d_off[k] / U, S + lay.s_off[k] / U, (const uint4 *)T->table.p, G, sg[k].log_m,
                          (int)sg[k].rows, T->cb, T->W, warps};
        warps += (unsigned)G * m;
        prod += msm_products(T->W, sg[k].log_m, !full) * ((double)sg[k].rows * m);
    }
    a.nseg = nseg;
    a.times_m = full ? 0 : 1;
    a.test_check = ctx->test_check;
    a.warps = warps;
    ctx->prof.begin(FK20_K_MSM, prod.alg, prod.exe, st);
    launch_msm(a, ctx->msm_threads, st);
    ctx->prof.end(st);
    CKL();
    if (full && ctx->fused_fft) {
        FusedPlan p{};
        unsigned widest = 0;
        prod = Work();
        for (int k = 0; k < nseg; k++) {
            const int log_m = sg[k].log_m, m = 1 << log_m, G = (int)((sg[k].rows + 31) / 32);
            p.seg[k] = FusedSeg{D + lay.d_off[k] / U, (unsigned *)((char *)ws.sync.p + SYNC_HDR + lay.r_off[k])};
            p.blk.G[k] = G;
            p.blk.log_m[k] = log_m;
            widest += (unsigned)G * (m / 2);
            for (int s = 0; s < log_m - 1; s++)
                prod += stage_products((int)sg[k].rows, log_m, s, 0) + stage_products((int)sg[k].rows, log_m, s + 1, 1);
            prod += Work((double)sg[k].rows * (m / 2) * ADD_P);
        }
        p.blk.nseg = nseg;
        fused_blocks_build(p.blk);
        p.next = (unsigned *)ws.sync.p;
        p.err = (int *)((char *)ws.sync.p + 128);
        p.epoch = 1;  // counters are cleared before every launch
        p.spin_limit = ctx->wait_limit;
        p.unpublished = ctx->unpublished;
        // persistent grid: the context's setting, or the caller's share of the SMs (server packs)
        int per_sm = ctx->fused_occupancy;
        const int want = fft_bps > 0 ? fft_bps : ctx->fft_blocks_per_sm;
        if (want > 0 && want < per_sm) per_sm = want;
        const unsigned max_blocks = (widest + FFT_WARPS - 1) / FFT_WARPS;
        p.blocks = (int)std::min<unsigned>((unsigned)(ctx->sms * per_sm), max_blocks);
        CK(cudaMemsetAsync(ws.sync.p, 0, SYNC_HDR + lay.r_bytes, st));
        ctx->prof.begin(FK20_K_FFT_FUSED, prod.alg, prod.exe, st);
        launch_g1_fused(p, st);
        ctx->prof.end(st);
        CKL();
        CK(cudaMemcpyAsync(ws.err_host, p.err, sizeof(int), cudaMemcpyDeviceToHost, st));
    } else if (full) {
        for (int k = 0; k < nseg; k++)
            CKR(run_hext_to_hfft(ctx->prof, D + lay.d_off[k] / U, (int)((sg[k].rows + 31) / 32), (int)sg[k].rows,
                                 sg[k].log_m, 0, st));
    }
    for (int k = 0; k < nseg; k++) {
        if (proofs) {  // compressed, data-availability order (kernels_out.cu)
            const double po = (double)sg[k].rows * (1 << sg[k].log_m) * PROOF_OUT_MP * MP;
            ctx->prof.begin(FK20_K_OUTPUT, po, po, st);
            launch_tile_to_proofs((uint8_t *)out, D + lay.d_off[k] / U, sg[k].out_off, (int)sg[k].rows,
                                  sg[k].log_m, st);
            ctx->prof.end(st);
            CKL();
        } else {
            CKR(output_launch(ctx->prof, (uint64_t *)out, D + lay.d_off[k] / U, sg[k].out_off, (int)sg[k].rows,
                              sg[k].log_m, 0, st));
        }
    }
    return 0;
}

// A ragged batch as segments, one per length (longest first): the offsets go
// to the workspace's device array through its pinned staging (no host wait
// unless the previous copy out of the staging is still pending).
int batch_segments(fk20_ctx *ctx, Workspace &ws, unsigned count, const unsigned *n, const size_t *poly_off,
                   const size_t *out_off, Seg *sg, int *nseg, cudaStream_t st) {
    CKR(ws.init());
    CKR(ws.stage_offsets(2 * (size_t)count));
    size_t *h = ws.offs_host;
    size_t at = 0;
    struct Part { int log_m; size_t first; unsigned rows; } parts[3];
    int np = 0;
    for (int log_m = 9; log_m >= 7; log_m--) {
        const unsigned nn = (unsigned)(L_COLS << (log_m - 1));
        Part pt{log_m, at, 0};
        for (unsigned j = 0; j < count; j++)
            if (n[j] == nn) { h[at++] = poly_off[j]; pt.rows++; }
        for (unsigned j = 0; j < count; j++)
            if (n[j] == nn) h[at++] = out_off[j];
        if (pt.rows) {
            if (!tables_for(ctx, log_m)->ready) return FK20_ENOSETUP;
            parts[np++] = pt;
        }
    }
    CKR(ws.offs.reserve(at * sizeof(size_t)));
    CK(cudaMemcpyAsync(ws.offs.p, h, at * sizeof(size_t), cudaMemcpyHostToDevice, st));
    CK(cudaEventRecord(ws.offs_done, st));
    const size_t *d = (const size_t *)ws.offs.p;
    for (int k = 0; k < np; k++)
        sg[k] = Seg{parts[k].log_m, parts[k].rows, d + parts[k].first, d + parts[k].first + parts[k].rows};
    *nseg = np;
    return 0;
}

int check_call(const void *out, const void *in, unsigned rows) {
    if (!out || !in) return FK20_EINVAL;
    if (rows == 0 || rows > MAX_ROWS) return FK20_EINVAL;
    if (((uintptr_t)out | (uintptr_t)in) & 15) return FK20_EINVAL;
    return 0;
}

int check_batch(const g1p_t *h_fft, const fr_t *polys, unsigned count, const unsigned *n, const size_t *poly_off,
                const size_t *out_off) {
    if (!h_fft || !polys || !n || !poly_off || !out_off || count == 0 || count > MAX_ROWS) return FK20_EINVAL;
    if (((uintptr_t)h_fft | (uintptr_t)polys) & 15) return FK20_EINVAL;
    for (unsigned j = 0; j < count; j++)
        if (log_m_for_n(n[j]) < 0) return FK20_EINVAL;
    return 0;
}

// ---- default context for the reference-signature entry points ---------------
std::mutex g_default_mu;
fk20_ctx *g_default[64];

int default_ctx(fk20_ctx **out) {
    int dev;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) { cudaGetLastError(); return FK20_ENODEV; }
    std::lock_guard<std::mutex> lk(g_default_mu);
    if (!g_default[dev]) {
        // FK20_WINDOW selects the default contexts' table window (8..15); unset = 10
        int w = 0;
        if (const char *e = getenv("FK20_WINDOW")) w = atoi(e);
        CKR(fk20_ctx_create(&g_default[dev], dev, w));
    }
    *out = g_default[dev];
    return 0;
}

int release_default(int dev) {
    if (dev < 0 || dev >= 64) return FK20_EINVAL;
    fk20_ctx *c = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_default_mu);
        c = g_default[dev];
        g_default[dev] = nullptr;
    }
    return c ? fk20_ctx_destroy(c) : 0;
}

// tables of the default context keyed by the content of xext_fft (caller holds ctx->mu)
int default_tables(fk20_ctx *ctx, const g1p_t *xext_fft, int log_m, cudaStream_t st) {
    const int m = 1 << log_m;
    unsigned long long fp = 0;
    CKR(fingerprint(ctx, xext_fft, (size_t)L_COLS * m * 18, &fp, st));
    Tables *T = tables_for(ctx, log_m);
    if (!T->ready || T->fingerprint != fp || T->cb != ctx->window) {
        CKR(build_tables(ctx, log_m, (const uint64_t *)xext_fft, st));
        T->fingerprint = fp;
    }
    return 0;
}

int setup2xext(fk20_ctx *ctx, g1p_t *xext_fft, const g1p_t *setup, unsigned n, cudaStream_t st) {
    const int log_m = log_m_for_n(n);
    const int m = 1 << log_m;
    CKR(ctx->D2.reserve(tile_bytes(1, m)));
    uint4 *D = (uint4 *)ctx->D2.p;
    launch_setup_to_tile(D, (const uint64_t *)setup, (int)n, log_m, st);
    CKL();
    for (int s = 0; s < log_m; s++) {
        launch_g1_stage(D, 1, log_m, s, 1, st);
        CKL();
    }
    launch_tile_to_ref((uint64_t *)xext_fft, D, nullptr, L_COLS, log_m, 0, st);
    CKL();
    return 0;
}

// natural-order G1 transforms of `count` rows of m points
int g1_transform(fk20_ctx *ctx, g1p_t *out, const g1p_t *in, int log_m, unsigned count, int inverse, cudaStream_t st) {
    const int m = 1 << log_m;
    const int G = (int)((count + 31) / 32);
    CKR(ctx->D2.reserve(tile_bytes(G, m)));
    uint4 *D = (uint4 *)ctx->D2.p;
    if (!inverse) {  // bit-reversed load, DIT forward -> natural order
        launch_ref_to_tile(D, (const uint64_t *)in, (int)count, G, log_m, 1, 0, st);
        CKL();
        for (int s = 0; s < log_m; s++) {
            launch_g1_stage(D, G, log_m, s, 1, st);
            CKL();
        }
        launch_tile_to_ref((uint64_t *)out, D, nullptr, (int)count, log_m, 0, st);
        CKL();
    } else {  // natural load, DIF inverse -> bit-reversed, times 1/m, reorder on store
        launch_ref_to_tile(D, (const uint64_t *)in, (int)count, G, log_m, 0, 0, st);
        CKL();
        for (int s = 0; s < log_m; s++) {
            launch_g1_stage(D, G, log_m, s, 0, st);
            CKL();
        }
        launch_g1_scale(D, G, log_m, 512 + log_m, st);
        CKL();
        launch_tile_to_ref((uint64_t *)out, D, nullptr, (int)count, log_m, 1, st);
        CKL();
    }
    return 0;
}

}  // namespace

// ============================================================================ C ABI
extern "C" {

const char *fk20_version(void) { return FK20_VERSION; }

int fk20_default_release(int device) { return release_default(device); }

int fk20_test_fail_allocations(int count) {
    if (count < 0) return FK20_EINVAL;
    g_fail_allocs.store(count);
    return 0;
}

int fk20_check_status(int *compiled) {
    if (compiled) *compiled = FK_CHECKED;
    if (cudaDeviceSynchronize() != cudaSuccess) return (int)cudaGetLastError();
    int v = check_take_msm();
    const int f = check_take_fft();
    return v ? v : f;
}

int fk20_ctx_create(fk20_ctx **out, int device, int window) {
    if (!out) return FK20_EINVAL;
    if (window == 0) window = 10;
    if (window < 8 || window > MAX_WINDOW) return FK20_EINVAL;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return FK20_ENODEV;
    }
    CKR(ensure_device(device));
    fk20_ctx *c = new fk20_ctx();
    c->device = device;
    c->window = window;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) == cudaSuccess) c->sms = prop.multiProcessorCount;
    {
        DeviceGuard dg(device);
        c->fused_occupancy = std::max(1, fused_blocks_per_sm());
        const int rc = c->ws.init();
        if (rc) {
            delete c;
            return rc;
        }
    }
    *out = c;
    return 0;
}

int fk20_ctx_set(fk20_ctx *ctx, int option, int value) {
    if (!ctx) return FK20_EINVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    switch (option) {
    case FK20_OPT_FUSED_FFT: ctx->fused_fft = value != 0; return 0;
    case FK20_OPT_MSM_THREADS:
        if (value != 64 && value != 128 && value != 256) return FK20_EINVAL;
        ctx->msm_threads = value;
        return 0;
    case FK20_OPT_FFT_BLOCKS_PER_SM:
        if (value < 0 || value > 64) return FK20_EINVAL;
        ctx->fft_blocks_per_sm = value;
        return 0;
    case FK20_OPT_WAIT_LIMIT:
        if (value < 0) return FK20_EINVAL;
        ctx->wait_limit = value ? (unsigned)value : FUSED_SPIN_LIMIT;
        return 0;
    case FK20_OPT_TEST_UNPUBLISHED_TASK:
        ctx->unpublished = value < 0 ? 0xffffffffu : (unsigned)value;
        return 0;
    case FK20_OPT_WINDOW:
        if (value < 8 || value > MAX_WINDOW) return FK20_EINVAL;
        ctx->window = value;
        return 0;
    case FK20_OPT_TEST_CHECK: ctx->test_check = value != 0; return 0;
    default: return FK20_EINVAL;
    }
}

int fk20_ctx_status(fk20_ctx *ctx) {
    if (!ctx) return FK20_EINVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    DeviceGuard dg(ctx->device);
    CK(cudaDeviceSynchronize());
    if (ctx->ws.err_host && *ctx->ws.err_host) {
        const int rc = launch_error(*ctx->ws.err_host);
        *ctx->ws.err_host = 0;
        return rc;
    }
    return 0;
}

int fk20_ctx_destroy(fk20_ctx *ctx) {
    if (!ctx) return FK20_EINVAL;
    {
        DeviceGuard dg(ctx->device);
        cudaDeviceSynchronize();
        for (auto &t : ctx->tab) t.table.release(), t.xext.release();
        ctx->commit.table.release();
        ctx->commit.part.release();
        ctx->ws.release();
        ctx->D2.release();
        ctx->scratch.release();
        ctx->xext.release();
        ctx->fp_dev.release();
        ctx->verify.release();
    }
    delete ctx;
    return 0;
}

int fk20_ctx_profile(fk20_ctx *ctx, int enable) {
    if (!ctx) return FK20_EINVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    DeviceGuard dg(ctx->device);
    ctx->prof.reset();
    ctx->prof.on = enable != 0;
    return 0;
}

int fk20_ctx_profile_read(fk20_ctx *ctx, int kind, double *ms, long *launches, double *products) {
    if (!ctx || kind < 0 || kind >= FK20_NKINDS) return FK20_EINVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    DeviceGuard dg(ctx->device);
    ctx->prof.collect();
    if (ms) *ms = ctx->prof.ms[kind];
    if (launches) *launches = ctx->prof.launches[kind];
    if (products) *products = ctx->prof.products[kind];
    return 0;
}

int fk20_ctx_profile_read_executed(fk20_ctx *ctx, int kind, double *products) {
    if (!ctx || kind < 0 || kind >= FK20_NKINDS || !products) return FK20_EINVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    DeviceGuard dg(ctx->device);
    ctx->prof.collect();
    *products = ctx->prof.executed[kind];
    return 0;
}

int fk20_program_cost(int index, int *dbl, int *add) {
    if (index < 0 || index >= NPROG || !dbl || !add) return FK20_EINVAL;
    const HostConsts &hc = host_consts();
    *dbl = hc.prog_dbl[index];
    *add = hc.prog_add[index];
    return 0;
}

size_t fk20_ctx_device_bytes(const fk20_ctx *ctx) {
    if (!ctx) return 0;
    size_t b = ctx->ws.bytes() + ctx->D2.bytes + ctx->scratch.bytes + ctx->xext.bytes;
    for (auto &t : ctx->tab) b += t.table.bytes + t.xext.bytes;
    b += ctx->commit.table.bytes + ctx->commit.part.bytes;
    return b;
}

int fk20_ctx_load_xext_fft(fk20_ctx *ctx, unsigned n, const g1p_t *xext_fft, void *stream) {
    const int log_m = log_m_for_n(n);
    if (!ctx || !xext_fft || log_m < 0) return FK20_EINVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    DeviceGuard dg(ctx->device);
    CKR(build_tables(ctx, log_m, (const uint64_t *)xext_fft, S_(stream)));
    tables_for(ctx, log_m)->fingerprint = 0;
    return 0;
}

int fk20_ctx_load_setup(fk20_ctx *ctx, unsigned n, const g1p_t *setup, void *stream) {
    const int log_m = log_m_for_n(n);
    if (!ctx || !setup || log_m < 0) return FK20_EINVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    DeviceGuard dg(ctx->device);
    const int m = 1 << log_m;
    CKR(ctx->xext.reserve((size_t)L_COLS * m * sizeof(g1p_t)));
    CKR(setup2xext(ctx, (g1p_t *)ctx->xext.p, setup, n, S_(stream)));
    CKR(build_tables(ctx, log_m, (const uint64_t *)ctx->xext.p, S_(stream)));
    tables_for(ctx, log_m)->fingerprint = 0;
    return 0;
}

int fk20_ctx_poly2h_fft(fk20_ctx *ctx, g1p_t *h_fft, const fr_t *polynomial, unsigned rows, unsigned n,
                        void *stream) {
    if (!ctx) return FK20_EINVAL;
    CKR(check_call(h_fft, polynomial, rows));
    const int log_m = log_m_for_n(n);
    if (log_m < 0) return FK20_EINVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    DeviceGuard dg(ctx->device);
    Tables *T = tables_for(ctx, log_m);
    if (!T->ready) return FK20_ENOSETUP;
    const Seg sg{log_m, rows, nullptr, nullptr};
    return run_segments(ctx, ctx->ws, &sg, 1, polynomial, h_fft, true, S_(stream));
}

int fk20_ctx_poly2hext_fft(fk20_ctx *ctx, g1p_t *hext_fft, const fr_t *polynomial, unsigned rows, unsigned n,
                           void *stream) {
    if (!ctx) return FK20_EINVAL;
    CKR(check_call(hext_fft, polynomial, rows));
    const int log_m = log_m_for_n(n);
    if (log_m < 0) return FK20_EINVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    DeviceGuard dg(ctx->device);
    Tables *T = tables_for(ctx, log_m);
    if (!T->ready) return FK20_ENOSETUP;
    const Seg sg{log_m, rows, nullptr, nullptr};
    return run_segments(ctx, ctx->ws, &sg, 1, polynomial, hext_fft, false, S_(stream));
}

int fk20_ctx_msm(fk20_ctx *ctx, g1p_t *hext_fft, const fr_t *tc_fft, unsigned rows, unsigned n, void *stream) {
    if (!ctx) return FK20_EINVAL;
    CKR(check_call(hext_fft, tc_fft, rows));
    const int log_m = log_m_for_n(n);
    if (log_m < 0) return FK20_EINVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    DeviceGuard dg(ctx->device);
    Tables *T = tables_for(ctx, log_m);
    if (!T->ready) return FK20_ENOSETUP;
    cudaStream_t st = S_(stream);
    const int m = 1 << log_m;
    const int G = (int)((rows + 31) / 32);
    CKR(ctx->ws.S.reserve(scal_bytes(G, m)));
    CKR(ctx->ws.D.reserve(tile_bytes(G, m)));
    launch_ref_to_scalars((uint4 *)ctx->ws.S.p, (const uint64_t *)tc_fft, (int)rows, log_m, st);
    CKL();
    CKR(msm_launch(ctx, T, (uint4 *)ctx->ws.D.p, (const uint4 *)ctx->ws.S.p, G, (int)rows, 1, st));
    CKR(output_launch(ctx->prof, (uint64_t *)hext_fft, (const uint4 *)ctx->ws.D.p, nullptr, (int)rows, log_m, 0, st));
    return 0;
}

int fk20_ctx_batch(fk20_ctx *ctx, g1p_t *h_fft, const fr_t *polys, unsigned count, const unsigned *n,
                   const size_t *poly_off, const size_t *out_off, void *stream) {
    if (!ctx) return FK20_EINVAL;
    CKR(check_batch(h_fft, polys, count, n, poly_off, out_off));
    std::lock_guard<std::mutex> lk(ctx->mu);
    DeviceGuard dg(ctx->device);
    cudaStream_t st = S_(stream);
    Seg sg[3];
    int nseg = 0;
    CKR(batch_segments(ctx, ctx->ws, count, n, poly_off, out_off, sg, &nseg, st));
    return run_segments(ctx, ctx->ws, sg, nseg, polys, h_fft, true, st);
}

int fk20_ctx_get(fk20_ctx *ctx, int option, int *value) {
    if (!ctx || !value) return FK20_EINVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    switch (option) {
    case FK20_OPT_FUSED_FFT: *value = ctx->fused_fft; return 0;
    case FK20_OPT_MSM_THREADS: *value = ctx->msm_threads; return 0;
    case FK20_OPT_WINDOW: *value = ctx->window; return 0;
    case FK20_OPT_FFT_BLOCKS_PER_SM: *value = ctx->fft_blocks_per_sm; return 0;
    case FK20_OPT_WAIT_LIMIT: *value = (int)ctx->wait_limit; return 0;
    case FK20_OPT_TEST_UNPUBLISHED_TASK: *value = ctx->unpublished == 0xffffffffu ? -1 : (int)ctx->unpublished; return 0;
    default: return FK20_EINVAL;
    }
}

}  // extern "C"

// ---------------------------------------------------------------- batch plans (CUDA graphs)
struct fk20_plan {
    fk20_ctx *ctx = nullptr;
    Workspace ws;
    cudaStream_t capture = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    unsigned gen[3] = {0, 0, 0};
    void release() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (capture) cudaStreamDestroy(capture);
        ws.release();
        exec = nullptr;
        graph = nullptr;
        capture = nullptr;
    }
};

namespace {

// the batch's launch sequence (offsets already on the device) captured into plan->graph
int capture_plan(fk20_plan *plan, g1p_t *h_fft, const fr_t *polys, const Seg *sg, int nseg) {
    fk20_ctx *ctx = plan->ctx;
    CKR(reserve_segments(ctx, plan->ws, sg, nseg, true));
    const bool prof_on = ctx->prof.on;
    ctx->prof.on = false;  // timing events cannot be replayed
    CK(cudaStreamBeginCapture(plan->capture, cudaStreamCaptureModeThreadLocal));
    const int rc = run_segments(ctx, plan->ws, sg, nseg, polys, h_fft, true, plan->capture);
    cudaGraph_t g = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(plan->capture, &g);
    ctx->prof.on = prof_on;
    if (rc) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        return rc;
    }
    CK(ec);
    plan->graph = g;
    CK(cudaGraphInstantiate(&plan->exec, g, 0));
    return 0;
}

}  // namespace

extern "C" {

int fk20_plan_create(fk20_plan **out, fk20_ctx *ctx, g1p_t *h_fft, const fr_t *polys, unsigned count,
                     const unsigned *n, const size_t *poly_off, const size_t *out_off) {
    if (!out || !ctx) return FK20_EINVAL;
    CKR(check_batch(h_fft, polys, count, n, poly_off, out_off));
    std::lock_guard<std::mutex> lk(ctx->mu);
    DeviceGuard dg(ctx->device);
    fk20_plan *plan = new fk20_plan();
    plan->ctx = ctx;
    int rc = plan->ws.init();
    if (!rc && cudaStreamCreateWithFlags(&plan->capture, cudaStreamNonBlocking) != cudaSuccess) rc = (int)cudaGetLastError();
    Seg sg[3];
    int nseg = 0;
    if (!rc) rc = batch_segments(ctx, plan->ws, count, n, poly_off, out_off, sg, &nseg, plan->capture);
    if (!rc) rc = (int)cudaStreamSynchronize(plan->capture);
    if (!rc) rc = capture_plan(plan, h_fft, polys, sg, nseg);
    if (rc) {
        plan->release();
        delete plan;
        return rc;
    }
    for (int k = 0; k < 3; k++) plan->gen[k] = ctx->tab[k].gen;
    *out = plan;
    return 0;
}

int fk20_plan_launch(fk20_plan *plan, void *stream) {
    if (!plan) return FK20_EINVAL;
    fk20_ctx *ctx = plan->ctx;
    std::lock_guard<std::mutex> lk(ctx->mu);
    DeviceGuard dg(ctx->device);
    for (int k = 0; k < 3; k++)
        if (plan->gen[k] != ctx->tab[k].gen) return FK20_ENOSETUP;
    if (*plan->ws.err_host) return launch_error(*plan->ws.err_host);
    CK(cudaGraphLaunch(plan->exec, S_(stream)));
    return 0;
}

int fk20_plan_destroy(fk20_plan *plan) {
    if (!plan) return FK20_EINVAL;
    {
        DeviceGuard dg(plan->ctx->device);
        cudaDeviceSynchronize();
        plan->release();
    }
    delete plan;
    return 0;
}

}  // extern "C"

// ---------------------------------------------------------------- autotuner
namespace {

size_t table_bytes_for(int log_m, int w) {
    const size_t W = (size_t)(GLV_TABLE_BITS + w - 1) / w;
    return (size_t)L_COLS * ((size_t)1 << log_m) * W * ((size_t)1 << (w - 1)) * 6 * sizeof(uint4);
}

struct Tuner {
    fk20_ctx *ctx;
    int log_m;
    unsigned rows;
    cudaStream_t st;
    const fr_t *poly;
    g1p_t *out;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    // average ms of one call after one untimed call
    int time(float *ms) {
        const Seg sg{log_m, rows, nullptr, nullptr};
        CKR(run_segments(ctx, ctx->ws, &sg, 1, poly, out, true, st));
        const int reps = 2;
        CK(cudaEventRecord(e0, st));
        for (int r = 0; r < reps; r++) CKR(run_segments(ctx, ctx->ws, &sg, 1, poly, out, true, st));
        CK(cudaEventRecord(e1, st));
        CK(cudaEventSynchronize(e1));
        if (*ctx->ws.err_host) {
            const int rc = launch_error(*ctx->ws.err_host);
            *ctx->ws.err_host = 0;
            return rc;
        }
        CK(cudaEventElapsedTime(ms, e0, e1));
        *ms /= reps;
        return 0;
    }
};

int autotune(fk20_ctx *ctx, int log_m, unsigned rows, size_t max_table_bytes, fk20_tune_result *res, cudaStream_t st) {
    Tables *T = tables_for(ctx, log_m);
    if (!T->ready) return FK20_ENOSETUP;
    const int m = 1 << log_m;
    const unsigned n = (unsigned)(m * L_COLS / 2);
    DevBuf poly, out;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    struct Release {  // the sample buffers and events go on every return path
        DevBuf &a, &b;
        cudaEvent_t &x, &y;
        ~Release() {
            a.release();
            b.release();
            if (x) cudaEventDestroy(x);
            if (y) cudaEventDestroy(y);
        }
    } release{poly, out, e0, e1};
    CKR(poly.reserve((size_t)rows * n * sizeof(fr_t)));
    CKR(out.reserve((size_t)rows * m * sizeof(g1p_t)));
    {  // sample coefficients: a SplitMix64 stream masked below 2^253 < r
        std::vector<uint64_t> h((size_t)rows * n * 4);
        uint64_t x = 0x5eed5eed5eedull;
        for (size_t i = 0; i < h.size(); i++) {
            uint64_t z = (x += 0x9E3779B97F4A7C15ull);
            z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
            z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
            h[i] = z ^ (z >> 31);
            if ((i & 3) == 3) h[i] &= (1ull << 61) - 1;
        }
        CK(cudaMemcpy(poly.p, h.data(), h.size() * sizeof(uint64_t), cudaMemcpyHostToDevice));
    }
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    Tuner tu{ctx, log_m, rows, st, (const fr_t *)poly.p, (g1p_t *)out.p, e0, e1};
    struct Cfg { int window, threads, bps, fused; };
    Cfg best{T->cb, ctx->msm_threads, ctx->fft_blocks_per_sm, ctx->fused_fft};
    float best_ms = 0;
    int rc = tu.time(&best_ms);
    const float ms_default = best_ms;
    auto apply = [&](const Cfg &c) {
        ctx->msm_threads = c.threads;
        ctx->fft_blocks_per_sm = c.bps;
        ctx->fused_fft = c.fused;
    };
    auto consider = [&](const Cfg &c) -> int {
        apply(c);
        float ms = 0;
        CKR(tu.time(&ms));
        if (ms < best_ms) best_ms = ms, best = c;
        apply(best);
        return 0;
    };
    // 1. table window, within the memory budget
    if (!rc) {
        size_t budget = max_table_bytes;
        if (!budget) {
            size_t fr = 0, tot = 0;
            CK(cudaMemGetInfo(&fr, &tot));
            const size_t margin = (size_t)4 << 30;
            budget = fr + T->table.bytes > margin ? fr + T->table.bytes - margin : 0;
        }
        const int w0 = T->cb;
        for (int w = 8; w <= MAX_WINDOW && !rc; w++) {
            if (w == w0 || table_bytes_for(log_m, w) > budget) continue;
            ctx->window = w;
            rc = build_tables(ctx, log_m, (const uint64_t *)T->xext.p, st);
            float ms = 0;
            if (!rc) rc = tu.time(&ms);
            if (!rc && ms < best_ms) best_ms = ms, best.window = w;
        }
        if (!rc && T->cb != best.window) {
            ctx->window = best.window;
            rc = build_tables(ctx, log_m, (const uint64_t *)T->xext.p, st);
        }
        ctx->window = best.window;
    }
    // 2. MSM block size, 3. persistent FFT grid, 4. fused vs staged FFT
    for (int t : {64, 128, 256})
        if (!rc && t != best.threads) rc = consider(Cfg{best.window, t, best.bps, best.fused});
    for (int b = 1; b <= ctx->fused_occupancy && !rc; b++)
        if (b != (best.bps ? best.bps : ctx->fused_occupancy)) rc = consider(Cfg{best.window, best.threads, b, 1});
    if (!rc) rc = consider(Cfg{best.window, best.threads, best.bps, best.fused ? 0 : 1});
    apply(best);
    cudaStreamSynchronize(st);
    if (rc) return rc;
    res->window = best.window;
    res->msm_threads = best.threads;
    res->fft_blocks_per_sm = best.bps;
    res->fused_fft = best.fused;
    res->ms = best_ms;
    res->ms_default = ms_default;
    return 0;
}

}  // namespace

extern "C" {

int fk20_ctx_autotune(fk20_ctx *ctx, unsigned n, unsigned rows, size_t max_table_bytes, fk20_tune_result *result,
                      void *stream) {
    const int log_m = log_m_for_n(n);
    if (!ctx || !result || log_m < 0 || rows == 0 || rows > 4096) return FK20_EINVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    DeviceGuard dg(ctx->device);
    return autotune(ctx, log_m, rows, max_table_bytes, result, S_(stream));
}

// ---------------------------------------------------------------- KZG commitments
int fk20_ctx_load_commit(fk20_ctx *ctx, unsigned n, const g1p_t *setup, int window, void *stream) {
    if (!ctx || !setup || n == 0 || n % COMMIT_CHUNK || n > (1u << 16)) return FK20_EINVAL;
    if (window == 0) window = 10;
    if (window < 8 || window > 13) return FK20_EINVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    DeviceGuard dg(ctx->device);
    cudaStream_t st = S_(stream);
    ctx->commit.n = 0;
    CKR(build_base_tables(ctx, ctx->commit.table, (const uint64_t *)setup, (int)n, window, -1, 255, st));
    CK(cudaStreamSynchronize(st));
    ctx->commit.cb = window;
    ctx->commit.W = (255 + window - 1) / window;
    ctx->commit.n = (int)n;
    return 0;
}

int fk20_ctx_commit(fk20_ctx *ctx, g1p_t *commitment, const fr_t *polynomial, unsigned rows, unsigned n,
                    void *stream) {
    if (!ctx) return FK20_EINVAL;
    CKR(check_call(commitment, polynomial, rows));
    if (n == 0 || n % COMMIT_CHUNK) return FK20_EINVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    DeviceGuard dg(ctx->device);
    if (!ctx->commit.n || (int)n > ctx->commit.n) return FK20_ENOSETUP;
    const int G = (int)((rows + 31) / 32);
    const int parts = commit_parts((int)rows, (int)n);
    CKR(ctx->commit.part.reserve(tile_bytes(G, parts)));
    const double terms = (double)rows * n * ctx->commit.W, sums = (double)rows * parts * ADD_P;
    ctx->prof.begin(FK20_K_MSM, terms * MADD_A + sums, terms * MADD_X + sums, S_(stream));
    launch_commit((uint64_t *)commitment, (uint4 *)ctx->commit.part.p, (const uint64_t *)polynomial,
                  (const uint4 *)ctx->commit.table.p, (int)rows, (int)n, ctx->commit.W, ctx->commit.cb, S_(stream));
    ctx->prof.end(S_(stream));
    CKL();
    return 0;
}

// ---------------------------------------------------------------- data-availability output
int fk20_g1p_compress_n(uint8_t *out, const g1p_t *p, size_t count, void *stream) {
    if (!out || !p || count == 0 || (((uintptr_t)out | (uintptr_t)p) & 15)) return FK20_EINVAL;
    CKR(current_device_ready());
    launch_g1p_compress(out, (const uint64_t *)p, count, S_(stream));
    CKL();
    return 0;
}

int fk20_h_fft2proofs(uint8_t *proofs, const g1p_t *h_fft, unsigned rows, unsigned n, void *stream) {
    const int log_m = log_m_for_n(n);
    if (log_m < 0) return FK20_EINVAL;
    CKR(check_call(proofs, h_fft, rows));
    CKR(current_device_ready());
    launch_h_fft_to_proofs(proofs, (const uint64_t *)h_fft, (int)rows, log_m, S_(stream));
    CKL();
    return 0;
}

int fk20_ctx_poly2proofs(fk20_ctx *ctx, uint8_t *proofs, const fr_t *polynomial, unsigned rows, unsigned n,
                         void *stream) {
    if (!ctx) return FK20_EINVAL;
    CKR(check_call(proofs, polynomial, rows));
    const int log_m = log_m_for_n(n);
    if (log_m < 0) return FK20_EINVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    DeviceGuard dg(ctx->device);
    if (!tables_for(ctx, log_m)->ready) return FK20_ENOSETUP;
    const Seg sg{log_m, rows, nullptr, nullptr};
    return run_segments(ctx, ctx->ws, &sg, 1, polynomial, proofs, true, S_(stream), true);
}

int fk20_ctx_batch_proofs(fk20_ctx *ctx, uint8_t *proofs, const fr_t *polys, unsigned count, const unsigned *n,
                          const size_t *poly_off, const size_t *out_off, void *stream) {
    if (!ctx) return FK20_EINVAL;
    CKR(check_batch((const g1p_t *)proofs, polys, count, n, poly_off, out_off));
    std::lock_guard<std::mutex> lk(ctx->mu);
    DeviceGuard dg(ctx->device);
    cudaStream_t st = S_(stream);
    Seg sg[3];
    int nseg = 0;
    CKR(batch_segments(ctx, ctx->ws, count, n, poly_off, out_off, sg, &nseg, st));
    return run_segments(ctx, ctx->ws, sg, nseg, polys, proofs, true, st, true);
}

// ---------------------------------------------------------------- reference entry points
int fk20_poly2h_fft(g1p_t *h_fft, const fr_t *polynomial, const g1p_t *xext_fft, unsigned rows) {
    if (!xext_fft) return FK20_EINVAL;
    CKR(check_call(h_fft, polynomial, rows));
    fk20_ctx *ctx;
    CKR(default_ctx(&ctx));
    {
        std::lock_guard<std::mutex> lk(ctx->mu);
        CKR(default_tables(ctx, xext_fft, 9, nullptr));
    }
    return fk20_ctx_poly2h_fft(ctx, h_fft, polynomial, rows, 4096, nullptr);
}

int fk20_poly2hext_fft(g1p_t *hext_fft, const fr_t *polynomial, const g1p_t *xext_fft, unsigned rows, void *stream) {
    if (!xext_fft) return FK20_EINVAL;
    CKR(check_call(hext_fft, polynomial, rows));
    fk20_ctx *ctx;
    CKR(default_ctx(&ctx));
    {
        std::lock_guard<std::mutex> lk(ctx->mu);
        CKR(default_tables(ctx, xext_fft, 9, S_(stream)));
    }
    return fk20_ctx_poly2hext_fft(ctx, hext_fft, polynomial, rows, 4096, stream);
}

int fk20_msm(g1p_t *hext_fft, const fr_t *tc_fft, const g1p_t *xext_fft, unsigned rows, void *stream) {
    if (!xext_fft) return FK20_EINVAL;
    CKR(check_call(hext_fft, tc_fft, rows));
    fk20_ctx *ctx;
    CKR(default_ctx(&ctx));
    {
        std::lock_guard<std::mutex> lk(ctx->mu);
        CKR(default_tables(ctx, xext_fft, 9, S_(stream)));
    }
    return fk20_ctx_msm(ctx, hext_fft, tc_fft, rows, 4096, stream);
}

int fk20_poly2toeplitz_coefficients(fr_t *tc, const fr_t *polynomial, unsigned rows, void *stream) {
    CKR(check_call(tc, polynomial, rows));
    CKR(current_device_ready());
    launch_toeplitz_ref((uint64_t *)tc, (const uint64_t *)polynomial, 4096, 9, rows, S_(stream));
    CKL();
    return 0;
}

int fk20_poly2toeplitz_coefficients_fft(fr_t *tc_fft, const fr_t *polynomial, unsigned rows, void *stream) {
    CKR(fk20_poly2toeplitz_coefficients(tc_fft, polynomial, rows, stream));
    return fr_fft_n(tc_fft, tc_fft, 9, rows * L_COLS, 0, stream);
}

int g1p_fft_n(g1p_t *output, const g1p_t *input, unsigned log_m, unsigned count, int inverse, void *stream) {
    if (log_m < 1 || log_m > 9) return FK20_EINVAL;
    CKR(check_call(output, input, count));
    fk20_ctx *ctx;
    CKR(default_ctx(&ctx));
    std::lock_guard<std::mutex> lk(ctx->mu);
    return g1_transform(ctx, output, input, (int)log_m, count, inverse, S_(stream));
}
int g1p_fft(g1p_t *output, const g1p_t *input, unsigned count, void *stream) {
    return g1p_fft_n(output, input, 9, count, 0, stream);
}
int g1p_ift(g1p_t *output, const g1p_t *input, unsigned count, void *stream) {
    return g1p_fft_n(output, input, 9, count, 1, stream);
}
int fk20_hext_fft2hext(g1p_t *hext, const g1p_t *hext_fft, unsigned rows, void *stream) {
    return g1p_ift(hext, hext_fft, rows, stream);
}
int fk20_h2h_fft(g1p_t *h_fft, const g1p_t *h, unsigned rows, void *stream) { return g1p_fft(h_fft, h, rows, stream); }

int fk20_hext2h(g1p_t *h, unsigned rows, void *stream) {
    CKR(check_call(h, h, rows));
    CKR(current_device_ready());
    launch_hext2h_ref((uint64_t *)h, (int)rows, 9, S_(stream));
    CKL();
    return 0;
}

int fk20_hext_fft2h(g1p_t *h, const g1p_t *hext_fft, unsigned rows, void *stream) {
    CKR(g1p_ift(h, hext_fft, rows, stream));
    return fk20_hext2h(h, rows, stream);
}

int fk20_hext_fft2h_fft(g1p_t *h_fft, const g1p_t *hext_fft, unsigned rows, void *stream) {
    CKR(check_call(h_fft, hext_fft, rows));
    fk20_ctx *ctx;
    CKR(default_ctx(&ctx));
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaStream_t st = S_(stream);
    const int log_m = 9, m = 512;
    const int G = (int)((rows + 31) / 32);
    CKR(ctx->D2.reserve(tile_bytes(G, m)));
    uint4 *D = (uint4 *)ctx->D2.p;
    launch_ref_to_tile(D, (const uint64_t *)hext_fft, (int)rows, G, log_m, 0, 0, st);
    CKL();
    CKR(run_hext_to_hfft(ctx->prof, D, G, (int)rows, log_m, 1, st));
    launch_tile_to_ref((uint64_t *)h_fft, D, nullptr, (int)rows, log_m, 0, st);
    CKL();
    return 0;
}

int fk20_setup2xext_fft(g1p_t *xext_fft, const g1p_t *setup, void *stream) {
    if (!xext_fft || !setup) return FK20_EINVAL;
    fk20_ctx *ctx;
    CKR(default_ctx(&ctx));
    std::lock_guard<std::mutex> lk(ctx->mu);
    return setup2xext(ctx, xext_fft, setup, 4096, S_(stream));
}

int fr_fft_n(fr_t *output, const fr_t *input, unsigned log_m, unsigned count, int inverse, void *stream) {
    if (log_m < 1 || log_m > 9) return FK20_EINVAL;
    CKR(check_call(output, input, count ? 1 : 0));
    if (count == 0) return FK20_EINVAL;
    CKR(current_device_ready());
    launch_fr_fft_ref((uint64_t *)output, (const uint64_t *)input, (int)log_m, count, inverse, S_(stream));
    CKL();
    return 0;
}
int fr_fft(fr_t *output, const fr_t *input, unsigned count, void *stream) { return fr_fft_n(output, input, 9, count, 0, stream); }
int fr_ift(fr_t *output, const fr_t *input, unsigned count, void *stream) { return fr_fft_n(output, input, 9, count, 1, stream); }

// ---------------------------------------------------------------- pairings
int fk20_pairing_check_n(uint8_t *ok, const g1p_t *a, const g2p_t *b, const g1p_t *c, const g2p_t *d, size_t count,
                         void *stream) {
    if (!ok || !a || !b || !c || !d || count == 0) return FK20_EINVAL;
    CKR(current_device_ready());
    launch_pairing(1, nullptr, ok, (const uint64_t *)a, (const uint64_t *)b, (const uint64_t *)c,
                   (const uint64_t *)d, count, S_(stream));
    CKL();
    return 0;
}

int fk20_ctx_check_proof_multi(fk20_ctx *ctx, uint8_t *ok, const g1p_t *commitment, const g1p_t *proof,
                               const fr_t *x, const fr_t *ys, unsigned l, const g2p_t *setup_g2, unsigned count,
                               void *stream) {
    if (!ctx || !ok || !commitment || !proof || !x || !ys || !setup_g2) return FK20_EINVAL;
    if (count == 0 || count > MAX_ROWS || l == 0 || l > COMMIT_CHUNK || (l & (l - 1))) return FK20_EINVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    DeviceGuard dg(ctx->device);
    if (ctx->commit.n < (int)COMMIT_CHUNK) return FK20_ENOSETUP;
    int log_l = 0;
    while ((1u << log_l) < l) log_l++;
    const int G = (int)((count + 31) / 32);
    const size_t poly_b = (size_t)count * COMMIT_CHUNK * sizeof(fr_t), xl_b = (size_t)count * sizeof(fr_t),
                 pt_b = (size_t)count * sizeof(g1p_t);
    CKR(ctx->verify.reserve(poly_b + xl_b + 3 * pt_b));
    CKR(ctx->commit.part.reserve(tile_bytes(G, commit_parts((int)count, (int)COMMIT_CHUNK))));
    char *base = (char *)ctx->verify.p;
    uint64_t *poly = (uint64_t *)base, *xl = (uint64_t *)(base + poly_b);
    uint64_t *I = (uint64_t *)(base + poly_b + xl_b), *T = I + 18 * (size_t)count, *A = T + 18 * (size_t)count;
    const cudaStream_t st = S_(stream);
    // I(X) over the coset and x^l; [I(s)]G1 with the commitment tables
    launch_interp(poly, xl, (const uint64_t *)x, (const uint64_t *)ys, log_l, count, st);
    launch_commit(I, (uint4 *)ctx->commit.part.p, poly, (const uint4 *)ctx->commit.table.p, (int)count,
                  (int)COMMIT_CHUNK, ctx->commit.W, ctx->commit.cb, st);
    // e(C - [I(s)] + [x^l] proof, G2) == e(proof, [s^l]G2)
    launch_g1_op(4, T, (const uint64_t *)proof, xl, count, st);
    launch_g1_op(3, A, (const uint64_t *)commitment, I, count, st);
    launch_g1_op(0, I, A, T, count, st);
    launch_pairing(1, nullptr, ok, I, (const uint64_t *)setup_g2, (const uint64_t *)proof,
                   (const uint64_t *)(setup_g2 + l), count, st, 3);
    CKL();
    return 0;
}

int fk20_pairing_n(fp_t *out, const g1p_t *a, const g2p_t *b, size_t count, void *stream) {
    if (!out || !a || !b || count == 0) return FK20_EINVAL;
    CKR(current_device_ready());
    launch_pairing(0, (uint64_t *)out, nullptr, (const uint64_t *)a, (const uint64_t *)b, nullptr, nullptr, count,
                   S_(stream));
    CKL();
    return 0;
}

int g2p_op_n(int op, g2p_t *out, const g2p_t *a, const void *b, size_t count, void *stream) {
    if (!a || op < 0 || op > 6 || count == 0) return FK20_EINVAL;
    if (op != 6 && !out) return FK20_EINVAL;
    if ((op == 0 || op == 3 || op == 4 || op == 6) && !b) return FK20_EINVAL;
    CKR(current_device_ready());
    launch_g2_op(op, (uint64_t *)out, (const uint64_t *)a, b, count, S_(stream));
    CKL();
    return 0;
}

// ---------------------------------------------------------------- element-wise
int fp_op_n(int op, fp_t *out, const fp_t *a, const fp_t *b, size_t count, void *stream) {
    if (!out || !a || op < 0 || op > 11 || count == 0) return FK20_EINVAL;
    if ((op == 0 || op == 2 || op == 3) && !b) return FK20_EINVAL;
    CKR(current_device_ready());
    launch_field_op(0, op, (uint64_t *)out, (const uint64_t *)a, (const uint64_t *)b, count, S_(stream));
    CKL();
    return 0;
}

int fr_op_n(int op, fr_t *out, const fr_t *a, const fr_t *b, size_t count, void *stream) {
    if (!out || !a || op < 0 || op > 11 || count == 0) return FK20_EINVAL;
    if ((op == 0 || op == 2 || op == 3) && !b) return FK20_EINVAL;
    CKR(current_device_ready());
    launch_field_op(1, op, (uint64_t *)out, (const uint64_t *)a, (const uint64_t *)b, count, S_(stream));
    CKL();
    return 0;
}

int g1p_op_n(int op, g1p_t *out, const g1p_t *a, const void *b, size_t count, void *stream) {
    if (!a || op < 0 || op > 6 || count == 0) return FK20_EINVAL;
    if (op != 6 && !out) return FK20_EINVAL;
    if ((op == 0 || op == 3 || op == 4 || op == 6) && !b) return FK20_EINVAL;
    CKR(current_device_ready());
    launch_g1_op(op, (uint64_t *)out, (const uint64_t *)a, b, count, S_(stream));
    CKL();
    return 0;
}

int fr_eq_n(uint8_t *eq, const fr_t *x, const fr_t *y, size_t count, void *stream) {
    if (!eq || !x || !y || count == 0) return FK20_EINVAL;
    CKR(current_device_ready());
    launch_fr_eq(eq, (const uint64_t *)x, (const uint64_t *)y, count, S_(stream));
    CKL();
    return 0;
}

int g1p_eq_n(uint8_t *eq, const g1p_t *p, const g1p_t *q, size_t count, void *stream) {
    if (!eq || !p || !q || count == 0) return FK20_EINVAL;
    CKR(current_device_ready());
    launch_g1p_eq(eq, (const uint64_t *)p, (const uint64_t *)q, count, S_(stream));
    CKL();
    return 0;
}

int g1a_fromG1p_n(g1a_t *a, const g1p_t *p, size_t count, void *stream) {
    if (!a || !p || count == 0) return FK20_EINVAL;
    CKR(current_device_ready());
    launch_g1a_from_g1p((uint64_t *)a, (const uint64_t *)p, count, S_(stream));
    CKL();
    return 0;
}

int fk20_bench_imad(uint32_t *sink, int blocks, int threads, int iters, void *stream) {
    if (!sink || blocks <= 0 || threads <= 0 || threads > 1024 || iters < 0) return FK20_EINVAL;
    CKR(current_device_ready());
    launch_bench_imad(sink, blocks, threads, iters, S_(stream));
    CKL();
    return 0;
}

int fk20_bench_field(int field, int sqr, uint32_t *data, size_t count, int iters, void *stream) {
    if (!data || count == 0 || iters < 0 || (field != 0 && field != 1)) return FK20_EINVAL;
    CKR(current_device_ready());
    launch_bench_field(field, sqr, data, count, iters, S_(stream));
    CKL();
    return 0;
}

}  // extern "C"

// ============================================================================ request server
// Continuous batching: one worker thread per server retires finished packs
// (copies their proofs to the callers' buffers), admits waiting requests into
// free slots as one mixed-length pack each, and otherwise sleeps until a
// request arrives or a pack's stream reaches its completion callback.
namespace {

using Clock = std::chrono::steady_clock;

struct Req {
    uint64_t ticket;
    const fr_t *poly;
    unsigned n;
    g1p_t *out;
    Clock::time_point t0;
};

struct Slot {
    cudaStream_t st = nullptr;
    cudaEvent_t done = nullptr;
    Workspace ws;
    DevBuf dpoly, dout;
    void *hpoly = nullptr, *hout = nullptr;  // pinned staging of the pack's inputs and outputs
    size_t hpoly_bytes = 0, hout_bytes = 0;
    std::vector<Req> reqs;     // the pack in flight (empty: the slot is free)
    std::vector<size_t> out_at;  // g1p_t offset of each request's proofs in hout
    int rc = 0;                // error of enqueueing the pack
    Clock::time_point t_form, t_enq;  // the pack was formed / fully enqueued
    size_t bytes() const { return ws.bytes() + dpoly.bytes + dout.bytes; }
};

int pinned_reserve(void **p, size_t *have, size_t need) {
    if (need <= *have) return 0;
    if (*p) cudaFreeHost(*p);
    *p = nullptr;
    *have = 0;
    if (cudaMallocHost(p, need) != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return FK20_ENOMEM;
    }
    *have = need;
    return 0;
}

// device bytes of a pack with cnt[k] requests of log_m = 7 + k
size_t pack_bytes(const unsigned cnt[3]) {
    size_t b = SYNC_HDR + 2 * sizeof(size_t) * (cnt[0] + cnt[1] + cnt[2]);
    for (int k = 0; k < 3; k++) {
        if (!cnt[k]) continue;
        const int m = 128 << k, G = (int)((cnt[k] + 31) / 32);
        b += (size_t)cnt[k] * ((size_t)m * 8 * sizeof(fr_t) + (size_t)m * sizeof(g1p_t));
        b += scal_bytes(G, m) + tile_bytes(G, m) + (size_t)G * m * sizeof(unsigned);
    }
    return b;
}

}  // namespace

namespace {
// engine 1: buffers of one cohort, sized at creation for cohort_rows rows of
// the longest length
struct CohortBuf {
    DevBuf S, D, ready, dpoly, dout;
    void *hpoly = nullptr, *hout = nullptr;
    cudaEvent_t msm_done = nullptr, out_done = nullptr;
};
// engine 1: requests of one length admitted together, proved as one segment
// of the persistent FFT launches; state 0 free, 1 formed and its inputs
// staged, 5 in the MSM batch, 2 in the FFT launches, 3 output copy enqueued
struct Cohort {
    int state = 0;
    int log_m = 0, rows = 0, G = 0;
    int stage = 0;       // first FFT stage not yet launched
    uint64_t order = 0;  // admission order (older cohorts first in a launch)
    int rc = 0;          // error of enqueueing its work
    std::vector<Req> reqs;
    Clock::time_point t_form, t_enq;
};
}  // namespace

struct fk20_server {
    fk20_ctx *ctx = nullptr;
    fk20_server_config cfg{};
    std::vector<Slot> slots;
    // engine 1 (cohorts)
    std::vector<CohortBuf> cbuf;
    std::vector<Cohort> cohort;
    cudaStream_t st_msm = nullptr, st_fft = nullptr;
    DevBuf hdr;                  // persistent-launch header: task counter at 0, error flag at 128
    int *iter_err = nullptr;     // pinned copy of the last launch's error flag
    cudaEvent_t iter_done = nullptr, msm_done = nullptr;
    bool iter_busy = false, msm_busy = false;
    uint64_t next_order = 1;
    Clock::time_point t_launch;  // the FFT launch in flight was enqueued
    double sum_msm_ms = 0, sum_launch_ms = 0;
    uint64_t launches = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Req> queue;
    std::unordered_set<uint64_t> live;             // submitted and not yet waited for
    std::unordered_map<uint64_t, int> finished;    // ticket -> status
    uint64_t next_ticket = 1;
    bool stop = false;
    std::atomic<bool> wake{false};  // set by the completion callback, which never takes `mu`
    std::thread worker;
    // statistics since the last reset
    std::vector<double> lat_ms;
    uint64_t proofs = 0, packs = 0, pack_rows = 0, rejected = 0, nomem = 0, cancelled = 0;
    double sum_wait_ms = 0, sum_enqueue_ms = 0, sum_run_ms = 0;  // where the latency goes
    Clock::time_point first, last;
    bool started = false;
};

namespace {

// Runs on CUDA's callback thread between a pack's last copy and its event:
// it must not block (the event, and so the slot, would never complete), so it
// only sets a flag and notifies; the worker's waits are bounded in case the
// notification lands before the worker sleeps.
void CUDART_CB pack_done_cb(void *p) {
    fk20_server *s = (fk20_server *)p;
    s->wake.store(true);
    s->cv_work.notify_all();
}

// inputs to pinned staging, one H2D copy, the segment pipeline, one D2H copy
int enqueue_pack(fk20_server *s, Slot &sl, bool latency) {
    const size_t cnt = sl.reqs.size();
    std::vector<unsigned> ns(cnt);
    std::vector<size_t> poly_off(cnt), out_off(cnt);
    size_t in = 0, out = 0;
    for (size_t i = 0; i < cnt; i++) {
        ns[i] = sl.reqs[i].n;
        poly_off[i] = in;
        out_off[i] = out;
        in += sl.reqs[i].n;
        out += sl.reqs[i].n / 8;
    }
    sl.out_at = out_off;
    CKR(pinned_reserve(&sl.hpoly, &sl.hpoly_bytes, in * sizeof(fr_t)));
    CKR(pinned_reserve(&sl.hout, &sl.hout_bytes, out * sizeof(g1p_t)));
    CKR(sl.dpoly.reserve(in * sizeof(fr_t)));
    CKR(sl.dout.reserve(out * sizeof(g1p_t)));
    for (size_t i = 0; i < cnt; i++)
        memcpy((fr_t *)sl.hpoly + poly_off[i], sl.reqs[i].poly, (size_t)sl.reqs[i].n * sizeof(fr_t));
    CK(cudaMemcpyAsync(sl.dpoly.p, sl.hpoly, in * sizeof(fr_t), cudaMemcpyHostToDevice, sl.st));
    {
        fk20_ctx *ctx = s->ctx;
        std::lock_guard<std::mutex> lk(ctx->mu);
        Seg sg[3];
        int nseg = 0;
        CKR(batch_segments(ctx, sl.ws, (unsigned)cnt, ns.data(), poly_off.data(), out_off.data(), sg, &nseg, sl.st));
        // The persistent FFT's blocks per SM.  Adaptive by default: a
        // latency-mode pack may fill the GPU, and the next pack's blocks take
        // over as its own retire (a pack alone finishes in about half the
        // time); a throughput-mode pack takes 1/slots of the SMs, so packs of
        // different slots run side by side and hide each other's dependency
        // waits.
        int share = ctx->fused_occupancy;
        if (s->cfg.fft_blocks_per_sm)
            share = std::min((int)s->cfg.fft_blocks_per_sm, ctx->fused_occupancy);
        else if (!latency)
            share = std::max(1, ctx->fused_occupancy / (int)s->slots.size());
        CKR(run_segments(ctx, sl.ws, sg, nseg, (const fr_t *)sl.dpoly.p, (g1p_t *)sl.dout.p, true, sl.st, false,
                         share));
    }
    CK(cudaMemcpyAsync(sl.hout, sl.dout.p, out * sizeof(g1p_t), cudaMemcpyDeviceToHost, sl.st));
    CK(cudaLaunchHostFunc(sl.st, pack_done_cb, s));
    CK(cudaEventRecord(sl.done, sl.st));
    return 0;
}

void server_main(fk20_server *s) {
    cudaSetDevice(s->ctx->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        // 1. retire finished packs
        bool retired = false;
        for (Slot &sl : s->slots) {
            if (sl.reqs.empty()) continue;
            int status = sl.rc;
            if (!status) {
                const cudaError_t q = cudaEventQuery(sl.done);
                if (q == cudaErrorNotReady) continue;
                if (q != cudaSuccess) {
                    cudaGetLastError();
                    status = (int)q;
                } else if (*sl.ws.err_host) {
                    status = launch_error(*sl.ws.err_host);
                    *sl.ws.err_host = 0;  // the next pack of this slot starts clean
                }
            }
            std::vector<Req> done;
            done.swap(sl.reqs);
            lk.unlock();
            if (!status)
                for (size_t i = 0; i < done.size(); i++)
                    memcpy(done[i].out, (const g1p_t *)sl.hout + sl.out_at[i], (size_t)(done[i].n / 8) * sizeof(g1p_t));
            const Clock::time_point now = Clock::now();
            lk.lock();
            for (const Req &r : done) {
                s->finished[r.ticket] = status;
                s->lat_ms.push_back(std::chrono::duration<double, std::milli>(now - r.t0).count());
                s->proofs += r.n / 8;
            }
            s->packs++;
            s->pack_rows += done.size();
            s->sum_run_ms += std::chrono::duration<double, std::milli>(now - sl.t_enq).count();
            s->last = now;
            sl.rc = 0;
            retired = true;
        }
        if (retired) s->cv_done.notify_all();
        // 2. admit waiting requests into a free slot
        Slot *fs = nullptr;
        size_t others = 0;
        for (Slot &sl : s->slots) {
            if (!fs && sl.reqs.empty()) fs = &sl;
            else others += sl.bytes();
        }
        if (fs && !s->queue.empty()) {
            // Latency mode while no more than latency_rows requests wait: the
            // pack takes them all.  Beyond that (a burst, or a load above what
            // latency-mode packs sustain), throughput mode: oldest first, up to
            // max_rows and the memory budget, and each length with 32 or more
            // in the pack keeps a multiple of 32 (a warp proves 32 rows of one
            // length; a partial group idles lanes): its youngest extra
            // requests go back to the head of the queue for the next pack.
            const bool latency = s->queue.size() <= s->cfg.latency_rows;
            const size_t cap = s->queue.size() > 2 * (size_t)s->cfg.max_rows ? s->cfg.burst_rows : s->cfg.max_rows;
            const bool more = s->queue.size() > cap;
            // Admission by device memory: the packs in flight and this one stay
            // within the budget, and whatever this pack adds to its slot's
            // buffers must be free on the device now (less a reserve for the
            // runtime and other users of the GPU).  A pack that fits the
            // slot's buffers takes no new memory, so the device is only asked
            // (once, without holding the server lock: submit must not wait on
            // the driver) when a pack would grow them.
            size_t limit = s->cfg.hbm_budget;
            bool asked = false;
            unsigned cnt[3] = {0, 0, 0};
            size_t q = 0;
            for (; q < s->queue.size() && fs->reqs.size() < cap; q++) {
                const Req r = s->queue[q];
                const int k = log_m_for_n(r.n) - 7;
                unsigned c2[3] = {cnt[0], cnt[1], cnt[2]};
                c2[k]++;
                const size_t need = std::max(fs->bytes(), pack_bytes(c2));
                if (need > fs->bytes() && !asked) {
                    asked = true;
                    size_t fr = 0, tot = 0;
                    lk.unlock();  // producers only append to the queue; the worker alone removes
                    const cudaError_t e = cudaMemGetInfo(&fr, &tot);
                    lk.lock();
                    if (e == cudaSuccess) {
                        const size_t reserve = (size_t)256 << 20;
                        limit = std::min(limit, others + fs->bytes() + (fr > reserve ? fr - reserve : 0));
                    } else {
                        cudaGetLastError();
                    }
                }
                if (others + need > limit) break;
                cnt[k]++;
                fs->reqs.push_back(r);
            }
            s->queue.erase(s->queue.begin(), s->queue.begin() + (long)q);
            if (more) {
                unsigned keep[3];
                for (int k = 0; k < 3; k++) keep[k] = cnt[k] >= 32 ? cnt[k] & ~31u : cnt[k];
                std::vector<Req> kept, back;
                for (size_t t = fs->reqs.size(); t-- > 0;) {
                    const int k = log_m_for_n(fs->reqs[t].n) - 7;
                    if (cnt[k] > keep[k]) {
                        back.push_back(fs->reqs[t]);
                        cnt[k]--;
                    } else {
                        kept.push_back(fs->reqs[t]);
                    }
                }
                fs->reqs.assign(kept.rbegin(), kept.rend());
                s->queue.insert(s->queue.begin(), back.rbegin(), back.rend());
            }
            if (fs->reqs.empty()) {
                // not even one request fits next to the packs in flight: wait
                // for one of them to complete; alone, it never fits
                bool busy = false;
                for (Slot &sl : s->slots) busy |= !sl.reqs.empty();
                if (!busy) {
                    s->finished[s->queue.front().ticket] = FK20_ENOMEM;
                    s->nomem++;
                    s->queue.pop_front();
                    s->cv_done.notify_all();
                } else {
                    s->cv_work.wait_for(lk, std::chrono::milliseconds(2), [&] { return s->wake.load() || s->stop; });
                    s->wake.store(false);
                }
                continue;
            } else {
                fs->t_form = Clock::now();
                for (const Req &r : fs->reqs)
                    s->sum_wait_ms += std::chrono::duration<double, std::milli>(fs->t_form - r.t0).count();
                lk.unlock();
                fs->rc = enqueue_pack(s, *fs, latency);
                fs->t_enq = Clock::now();
                lk.lock();
                s->sum_enqueue_ms += std::chrono::duration<double, std::milli>(fs->t_enq - fs->t_form).count();
                continue;
            }
        }
        bool busy = false;
        for (Slot &sl : s->slots) busy |= !sl.reqs.empty();
        if (s->stop && s->queue.empty() && !busy) break;
        // 3. sleep until a request arrives or a pack completes (bounded, as a backstop)
        s->cv_work.wait_for(lk, std::chrono::milliseconds(busy ? 2 : 50), [&] {
            if (s->wake.load() || s->stop) return true;
            if (s->queue.empty()) return false;
            for (Slot &sl : s->slots)
                if (sl.reqs.empty()) return true;
            return false;
        });
        s->wake.store(false);
    }
}

// ---------------------------------------------------------------- engine 1: cohorts
// Continuous batching at FFT-stage granularity.  The waiting requests of one
// length become a cohort (one segment of up to cohort_rows rows) as soon as a
// 32-row group is full or the oldest has waited form_ms.  Its inputs are
// staged and its toeplitz + MSM run on their own stream; once that is done
// the cohort joins the persistent FFT launches, each of which advances every
// cohort in flight by stages_per_launch stages (a stage window per segment:
// the readiness counters and tiles carry over from launch to launch, with the
// same epoch, so a window's first stage finds its inputs ready).  A cohort
// whose last stage ran gets its output kernel and copy behind that launch.
// One FFT launch is in flight at a time; the MSMs of new cohorts run beside
// it.

// inputs of a formed cohort into its pinned staging (host copies only)
void cohort_stage(Cohort &c, const CohortBuf &b) {
    const size_t n = (size_t)8 << c.log_m;
    for (size_t i = 0; i < c.reqs.size(); i++)
        memcpy((fr_t *)b.hpoly + i * n, c.reqs[i].poly, n * sizeof(fr_t));
}

// The new cohorts' inputs, toeplitz + Fr FFTs and ONE MSM launch over all of
// them, on the MSM stream (beside the FFT launches); `msm_done` follows it.
int cohort_msm(fk20_server *s, const std::vector<int> &fresh) {
    fk20_ctx *ctx = s->ctx;
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaStream_t st = s->st_msm;
    MsmArgs a{};
    unsigned warps = 0;
    for (size_t k = 0; k < fresh.size(); k++) {
        const Cohort &c = s->cohort[fresh[k]];
        const CohortBuf &b = s->cbuf[fresh[k]];
        const int m = 1 << c.log_m, n = m * 8;
        Tables *T = tables_for(ctx, c.log_m);
        CK(cudaMemcpyAsync(b.dpoly.p, b.hpoly, (size_t)c.rows * n * sizeof(fr_t), cudaMemcpyHostToDevice, st));
        launch_tc_fft((uint4 *)b.S.p, (const uint64_t *)b.dpoly.p, nullptr, n, c.log_m, (unsigned)c.rows, st);
        CKL();
        CK(cudaMemsetAsync(b.ready.p, 0, (size_t)c.G * m * sizeof(unsigned), st));
        a.seg[k] = MsmSeg{(uint4 *)b.D.p, (const uint4 *)b.S.p, (const uint4 *)T->table.p, c.G, c.log_m, c.rows,
                          T->cb, T->W, warps};
        warps += (unsigned)c.G << c.log_m;
    }
    a.nseg = (int)fresh.size();
    a.times_m = 0;
    a.test_check = ctx->test_check;
    a.warps = warps;
    launch_msm(a, ctx->msm_threads, st);
    CKL();
    CK(cudaEventRecord(s->msm_done, st));
    CK(cudaLaunchHostFunc(st, pack_done_cb, s));
    return 0;
}

// One persistent FFT launch on the FFT stream that advances every cohort in
// `act` (oldest first) by up to stages_per_launch stages, then the outputs of
// the cohorts that finished.
int cohort_launch(fk20_server *s, const std::vector<int> &act) {
    fk20_ctx *ctx = s->ctx;
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaStream_t st = s->st_fft;
    FusedPlan p{};
    unsigned widest = 0;
    for (size_t k = 0; k < act.size(); k++) {
        Cohort &c = s->cohort[act[k]];
        const CohortBuf &b = s->cbuf[act[k]];
        const int m = 1 << c.log_m, total = 2 * c.log_m - 1;
        p.seg[k] = FusedSeg{(uint4 *)b.D.p, (unsigned *)b.ready.p};
        p.blk.G[k] = c.G;
        p.blk.log_m[k] = c.log_m;
        p.blk.s_lo[k] = (unsigned char)c.stage;
        p.blk.s_hi[k] = (unsigned char)std::min(total, c.stage + (int)s->cfg.stages_per_launch);
        widest += (unsigned)c.G * (m / 2);
    }
    p.blk.nseg = (int)act.size();
    fused_blocks_build(p.blk);
    p.next = (unsigned *)s->hdr.p;
    p.err = (int *)((char *)s->hdr.p + 128);
    p.epoch = 1;  // fixed for a cohort's life: its counters carry over between launches
    p.spin_limit = ctx->wait_limit;
    p.unpublished = ctx->unpublished;
    const unsigned max_blocks = (widest + FFT_WARPS - 1) / FFT_WARPS;
    p.blocks = (int)std::min<unsigned>((unsigned)(ctx->sms * ctx->fused_occupancy), max_blocks);
    CK(cudaMemsetAsync(s->hdr.p, 0, SYNC_HDR, st));
    launch_g1_fused(p, st);
    CKL();
    CK(cudaMemcpyAsync(s->iter_err, p.err, sizeof(int), cudaMemcpyDeviceToHost, st));
    for (size_t k = 0; k < act.size(); k++) {
        Cohort &c = s->cohort[act[k]];
        const CohortBuf &b = s->cbuf[act[k]];
        c.stage = p.blk.s_hi[k];
        if (c.stage < 2 * c.log_m - 1) continue;
        const int m = 1 << c.log_m;
        launch_tile_to_ref((uint64_t *)b.dout.p, (const uint4 *)b.D.p, nullptr, c.rows, c.log_m, 0, st);
        CKL();
        CK(cudaMemcpyAsync(b.hout, b.dout.p, (size_t)c.rows * m * sizeof(g1p_t), cudaMemcpyDeviceToHost, st));
        CK(cudaEventRecord(b.out_done, st));
        c.state = 3;
    }
    CK(cudaEventRecord(s->iter_done, st));
    CK(cudaLaunchHostFunc(st, pack_done_cb, s));
    return 0;
}

// a cohort's requests finish with `status` (caller holds the server lock)
void cohort_finish(fk20_server *s, Cohort &c, int status, Clock::time_point now) {
    for (const Req &r : c.reqs) {
        s->finished[r.ticket] = status;
        if (!status) {
            s->lat_ms.push_back(std::chrono::duration<double, std::milli>(now - r.t0).count());
            s->proofs += r.n / 8;
        }
    }
    s->packs++;
    s->pack_rows += c.reqs.size();
    s->sum_run_ms += std::chrono::duration<double, std::milli>(now - c.t_enq).count();
    s->last = now;
    c.reqs.clear();
    c.state = 0;
    c.rc = 0;
}

void server_main_cohorts(fk20_server *s) {
    cudaSetDevice(s->ctx->device);
    const int NC = (int)s->cohort.size();
    const int rows_max = (int)s->cfg.cohort_rows;
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        bool progress = false;
        // 1. the FFT launch in flight
        if (s->iter_busy) {
            const cudaError_t q = cudaEventQuery(s->iter_done);
            if (q != cudaErrorNotReady) {
                s->iter_busy = false;
                s->launches++;
                s->sum_launch_ms += std::chrono::duration<double, std::milli>(Clock::now() - s->t_launch).count();
                int status = 0;
                if (q != cudaSuccess) {
                    cudaGetLastError();
                    status = (int)q;
                } else if (*s->iter_err) {
                    status = launch_error(*s->iter_err);
                    *s->iter_err = 0;
                }
                if (status) {  // every cohort that was in the launch has invalid tiles
                    const Clock::time_point now = Clock::now();
                    for (Cohort &c : s->cohort)
                        if (c.state == 2 || c.state == 3) cohort_finish(s, c, status, now);
                    s->cv_done.notify_all();
                }
                progress = true;
            }
        }
        // 2. outputs copied: hand the proofs to the callers
        for (int i = 0; i < NC; i++) {
            Cohort &c = s->cohort[i];
            if (c.state != 3) continue;
            const cudaError_t q = cudaEventQuery(s->cbuf[i].out_done);
            if (q == cudaErrorNotReady) continue;
            int status = 0;
            if (q != cudaSuccess) {
                cudaGetLastError();
                status = (int)q;
            }
            std::vector<Req> done;
            done.swap(c.reqs);
            c.state = 4;  // copying out: not free yet
            lk.unlock();
            if (!status) {
                const size_t per = (size_t)(1 << c.log_m);
                for (size_t k = 0; k < done.size(); k++)
                    memcpy(done[k].out, (const g1p_t *)s->cbuf[i].hout + k * per, per * sizeof(g1p_t));
            }
            const Clock::time_point now = Clock::now();
            lk.lock();
            c.reqs.swap(done);
            cohort_finish(s, c, status, now);
            s->cv_done.notify_all();
            progress = true;
        }
        // 4. new cohorts: per length (longest first), whole 32-row groups, or
        // what waits once its oldest request has waited form_ms (or at shutdown)
        const Clock::time_point now = Clock::now();
        for (int L = 9; L >= 7 && !s->queue.empty(); L--) {
            int freei = -1;
            for (int i = 0; i < NC; i++)
                if (s->cohort[i].state == 0) {
                    freei = i;
                    break;
                }
            if (freei < 0) break;
            size_t count = 0;
            double oldest_ms = 0;
            for (const Req &r : s->queue)
                if (log_m_for_n(r.n) == L) {
                    if (!count) oldest_ms = std::chrono::duration<double, std::milli>(now - r.t0).count();
                    count++;
                }
            if (!count) continue;
            const bool late = s->stop || oldest_ms >= (double)s->cfg.form_ms;
            size_t take = std::min(count, (size_t)rows_max);
            if (!late) take = take / 32 * 32;
            if (!take) continue;
            Cohort &c = s->cohort[freei];
            c.reqs.clear();
            std::deque<Req> rest;
            for (const Req &r : s->queue) {
                if (c.reqs.size() < take && log_m_for_n(r.n) == L) c.reqs.push_back(r);
                else rest.push_back(r);
            }
            s->queue.swap(rest);
            c.log_m = L;
            c.rows = (int)c.reqs.size();
            c.G = (c.rows + 31) / 32;
            c.stage = 0;
            c.order = s->next_order++;
            c.state = 1;
            c.t_form = Clock::now();
            for (const Req &r : c.reqs)
                s->sum_wait_ms += std::chrono::duration<double, std::milli>(c.t_form - r.t0).count();
            lk.unlock();
            cohort_stage(c, s->cbuf[freei]);
            c.t_enq = Clock::now();
            lk.lock();
            s->sum_enqueue_ms += std::chrono::duration<double, std::milli>(c.t_enq - c.t_form).count();
            progress = true;
        }
        // 5. the MSM batch in flight: done -> its cohorts join the FFT launches
        if (s->msm_busy) {
            const cudaError_t q = cudaEventQuery(s->msm_done);
            if (q != cudaErrorNotReady) {
                s->msm_busy = false;
                const Clock::time_point t = Clock::now();
                for (Cohort &c : s->cohort) {
                    if (c.state != 5) continue;
                    if (q != cudaSuccess) {
                        cohort_finish(s, c, (int)q, t);
                    } else {
                        c.state = 2;
                        s->sum_msm_ms += std::chrono::duration<double, std::milli>(t - c.t_enq).count();
                    }
                }
                if (q != cudaSuccess) {
                    cudaGetLastError();
                    s->cv_done.notify_all();
                }
                progress = true;
            }
        }
        // 6. the next MSM batch: every staged cohort
        if (!s->msm_busy) {
            std::vector<int> fresh;
            for (int i = 0; i < NC; i++)
                if (s->cohort[i].state == 1) fresh.push_back(i);
            if (!fresh.empty()) {
                for (int i : fresh) s->cohort[i].state = 5;
                s->msm_busy = true;
                lk.unlock();
                const int rc = cohort_msm(s, fresh);
                lk.lock();
                if (rc) {
                    s->msm_busy = false;
                    const Clock::time_point t = Clock::now();
                    for (int i : fresh) cohort_finish(s, s->cohort[i], rc, t);
                    s->cv_done.notify_all();
                }
                progress = true;
            }
        }
        // 7. the next FFT launch over the cohorts in the FFT stages, oldest first
        if (!s->iter_busy) {
            std::vector<int> act;
            for (int i = 0; i < NC; i++)
                if (s->cohort[i].state == 2) act.push_back(i);
            std::sort(act.begin(), act.end(),
                      [&](int x, int y) { return s->cohort[x].order < s->cohort[y].order; });
            if (!act.empty()) {
                s->iter_busy = true;
                s->t_launch = Clock::now();
                lk.unlock();
                const int rc = cohort_launch(s, act);
                lk.lock();
                if (rc) {  // nothing of it reached the GPU in a usable state
                    s->iter_busy = false;
                    const Clock::time_point t = Clock::now();
                    for (int i : act) cohort_finish(s, s->cohort[i], rc, t);
                    s->cv_done.notify_all();
                }
                progress = true;
            }
        }
        bool busy = s->iter_busy || s->msm_busy;
        for (const Cohort &c : s->cohort) busy |= c.state != 0;
        if (s->stop && s->queue.empty() && !busy) break;
        if (progress) continue;
        // sleep until a request arrives or a stream reaches its callback;
        // bounded, to re-check the formation deadline
        s->cv_work.wait_for(lk, std::chrono::milliseconds(1), [&] { return s->wake.load() || s->stop; });
        s->wake.store(false);
    }
}

void server_free(fk20_server *s) {
    DeviceGuard dg(s->ctx->device);
    if (s->st_msm) cudaStreamSynchronize(s->st_msm);
    if (s->st_fft) cudaStreamSynchronize(s->st_fft);
    for (CohortBuf &b : s->cbuf) {
        b.S.release();
        b.D.release();
        b.ready.release();
        b.dpoly.release();
        b.dout.release();
        if (b.hpoly) cudaFreeHost(b.hpoly);
        if (b.hout) cudaFreeHost(b.hout);
        if (b.msm_done) cudaEventDestroy(b.msm_done);
        if (b.out_done) cudaEventDestroy(b.out_done);
    }
    s->cbuf.clear();
    s->hdr.release();
    if (s->iter_err) cudaFreeHost(s->iter_err);
    if (s->iter_done) cudaEventDestroy(s->iter_done);
    if (s->msm_done) cudaEventDestroy(s->msm_done);
    if (s->st_msm) cudaStreamDestroy(s->st_msm);
    if (s->st_fft) cudaStreamDestroy(s->st_fft);
    s->iter_err = nullptr;
    s->iter_done = s->msm_done = nullptr;
    s->st_msm = s->st_fft = nullptr;
    for (Slot &sl : s->slots) {
        if (sl.st) cudaStreamSynchronize(sl.st);
        sl.ws.release();
        sl.dpoly.release();
        sl.dout.release();
        if (sl.hpoly) cudaFreeHost(sl.hpoly);
        if (sl.hout) cudaFreeHost(sl.hout);
        if (sl.done) cudaEventDestroy(sl.done);
        if (sl.st) cudaStreamDestroy(sl.st);
    }
    s->slots.clear();
}

}  // namespace

extern "C" {

int fk20_server_create(fk20_server **out, fk20_ctx *ctx, const fk20_server_config *cfg) {
    if (!out || !ctx) return FK20_EINVAL;
    fk20_server_config c = cfg ? *cfg : fk20_server_config{};
    if (!c.max_rows) c.max_rows = 160;
    if (!c.latency_rows) c.latency_rows = c.max_rows;
    if (c.latency_rows > c.max_rows) return FK20_EINVAL;
    if (!c.slots) c.slots = 2;
    if (!c.max_queue) c.max_queue = 1u << 16;
    if (c.max_rows > 4096 || c.slots > 8) return FK20_EINVAL;
    if (!c.burst_rows) c.burst_rows = std::min(4096u, c.max_rows + c.max_rows * 2 / 5);
    if (c.burst_rows < c.max_rows || c.burst_rows > 4096) return FK20_EINVAL;
    if (c.engine > 1) return FK20_EINVAL;
    if (!c.cohort_rows) c.cohort_rows = 64;
    if (!c.cohorts) c.cohorts = 16;
    if (!c.form_ms) c.form_ms = 25;
    if (!c.stages_per_launch) c.stages_per_launch = 3;
    if (c.cohort_rows < 32 || c.cohort_rows > 256 || c.cohorts > (unsigned)MAX_SEGS || c.stages_per_launch > 17)
        return FK20_EINVAL;
    fk20_server *s = new fk20_server();
    s->ctx = ctx;
    if (c.engine == 1) {
        // cohort buffers for cohort_rows rows of the longest length, all at creation
        DeviceGuard dg(ctx->device);
        int rc = 0;
        const int m = 512, n = 4096, G = (int)((c.cohort_rows + 31) / 32);
        s->cbuf.resize(c.cohorts);
        s->cohort.resize(c.cohorts);
        if (cudaStreamCreateWithFlags(&s->st_msm, cudaStreamNonBlocking) != cudaSuccess ||
            cudaStreamCreateWithFlags(&s->st_fft, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&s->iter_done, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&s->msm_done, cudaEventDisableTiming) != cudaSuccess)
            rc = (int)cudaGetLastError();
        if (!rc && cudaMallocHost(&s->iter_err, sizeof(int)) != cudaSuccess) {
            cudaGetLastError();
            rc = FK20_ENOMEM;
        }
        if (!rc) {
            *s->iter_err = 0;
            rc = s->hdr.reserve(SYNC_HDR);
        }
        for (CohortBuf &b : s->cbuf) {
            if (rc) break;
            const size_t in_b = (size_t)c.cohort_rows * n * sizeof(fr_t), out_b = (size_t)c.cohort_rows * m * sizeof(g1p_t);
            rc = b.S.reserve(scal_bytes(G, m));
            if (!rc) rc = b.D.reserve(tile_bytes(G, m));
            if (!rc) rc = b.ready.reserve((size_t)G * m * sizeof(unsigned));
            if (!rc) rc = b.dpoly.reserve(in_b);
            if (!rc) rc = b.dout.reserve(out_b);
            if (!rc && (cudaMallocHost(&b.hpoly, in_b) != cudaSuccess || cudaMallocHost(&b.hout, out_b) != cudaSuccess)) {
                cudaGetLastError();
                rc = FK20_ENOMEM;
            }
            if (!rc && (cudaEventCreateWithFlags(&b.msm_done, cudaEventDisableTiming) != cudaSuccess ||
                        cudaEventCreateWithFlags(&b.out_done, cudaEventDisableTiming) != cudaSuccess))
                rc = (int)cudaGetLastError();
        }
        if (rc) {
            server_free(s);
            delete s;
            return rc;
        }
        s->cfg = c;
        s->worker = std::thread(server_main_cohorts, s);
        *out = s;
        return 0;
    }
    {
        DeviceGuard dg(ctx->device);
        if (!c.hbm_budget) {
            size_t fr = 0, tot = 0;
            if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
                cudaGetLastError();
                delete s;
                return FK20_ENODEV;
            }
            c.hbm_budget = fr / 2;
        }
        s->slots.resize(c.slots);
        int rc = 0;
        // Size every slot for a full pack now (burst_rows requests of the
        // longest length, plus a partial group per length) when that fits the
        // budget: growing a buffer later would synchronise the device and
        // stall the other slots' packs.
        const unsigned cap = c.burst_rows;
        const unsigned full[3] = {32, 32, cap + 32};
        const bool presize = pack_bytes(full) * c.slots <= c.hbm_budget;
        for (Slot &sl : s->slots) {
            if (!rc && cudaStreamCreateWithFlags(&sl.st, cudaStreamNonBlocking) != cudaSuccess) rc = (int)cudaGetLastError();
            if (!rc && cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming) != cudaSuccess) rc = (int)cudaGetLastError();
            if (!rc) rc = sl.ws.init();
            if (!rc && presize) {
                const size_t in_b = (size_t)(cap + 64) * 4096 * sizeof(fr_t);
                const size_t out_b = (size_t)(cap + 64) * 512 * sizeof(g1p_t);
                const Seg sg[3] = {{7, 32, nullptr, nullptr}, {8, 32, nullptr, nullptr},
                                   {9, cap + 32, nullptr, nullptr}};
                rc = sl.dpoly.reserve(in_b);
                if (!rc) rc = sl.dout.reserve(out_b);
                if (!rc) rc = pinned_reserve(&sl.hpoly, &sl.hpoly_bytes, in_b);
                if (!rc) rc = pinned_reserve(&sl.hout, &sl.hout_bytes, out_b);
                if (!rc) rc = sl.ws.stage_offsets(2 * (size_t)(cap + 64));
                if (!rc) rc = sl.ws.offs.reserve(2 * (size_t)(cap + 64) * sizeof(size_t));
                if (!rc) {
                    SegLayout lay;
                    for (int k = 0; k < 3 && !rc; k++) {
                        const int m = 1 << sg[k].log_m, G = (int)((sg[k].rows + 31) / 32);
                        lay.s_bytes += scal_bytes(G, m);
                        lay.d_bytes += tile_bytes(G, m);
                        lay.r_bytes += (size_t)G * m * sizeof(unsigned);
                    }
                    rc = sl.ws.S.reserve(lay.s_bytes);
                    if (!rc) rc = sl.ws.D.reserve(lay.d_bytes);
                    if (!rc) rc = sl.ws.sync.reserve(SYNC_HDR + lay.r_bytes);
                }
            }
        }
        if (rc) {
            server_free(s);
            delete s;
            return rc;
        }
    }
    s->cfg = c;
    s->worker = std::thread(server_main, s);
    *out = s;
    return 0;
}

int fk20_server_submit(fk20_server *s, const fr_t *poly, unsigned n, g1p_t *h_fft, uint64_t *ticket) {
    if (!s || !poly || !h_fft || !ticket) return FK20_EINVAL;
    const int log_m = log_m_for_n(n);
    if (log_m < 0) return FK20_EINVAL;
    if (!tables_for(s->ctx, log_m)->ready) return FK20_ENOSETUP;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) return FK20_EINVAL;
        if (s->queue.size() >= s->cfg.max_queue) {
            s->rejected++;
            return FK20_EAGAIN;
        }
        const Clock::time_point now = Clock::now();
        const uint64_t t = s->next_ticket++;
        s->queue.push_back(Req{t, poly, n, h_fft, now});
        s->live.insert(t);
        if (!s->started) s->first = now, s->started = true;
        *ticket = t;
    }
    s->cv_work.notify_all();
    return 0;
}

int fk20_server_wait(fk20_server *s, uint64_t ticket, int timeout_ms) {
    if (!s) return FK20_EINVAL;
    std::unique_lock<std::mutex> lk(s->mu);
    if (!s->live.count(ticket)) return FK20_EINVAL;
    auto ready = [&] { return s->finished.count(ticket) != 0; };
    if (timeout_ms < 0) s->cv_done.wait(lk, ready);
    else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) return FK20_EAGAIN;
    const int status = s->finished[ticket];
    s->finished.erase(ticket);
    s->live.erase(ticket);
    return status;
}

int fk20_server_cancel(fk20_server *s, uint64_t ticket) {
    if (!s) return FK20_EINVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    if (!s->live.count(ticket) || s->finished.count(ticket)) return FK20_EINVAL;
    for (auto it = s->queue.begin(); it != s->queue.end(); ++it) {
        if (it->ticket != ticket) continue;
        s->queue.erase(it);  // never packed: the worker will not touch its buffers
        s->finished[ticket] = FK20_ECANCELED;
        s->cancelled++;
        s->cv_done.notify_all();
        return 0;
    }
    return FK20_EAGAIN;  // in a pack on the GPU: it completes normally
}

int fk20_server_get_stats(fk20_server *s, fk20_server_stats *out) {
    if (!s || !out) return FK20_EINVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    fk20_server_stats st{};
    std::vector<double> v = s->lat_ms;
    std::sort(v.begin(), v.end());
    st.requests = v.size();
    st.proofs = s->proofs;
    st.packs = s->packs;
    if (!v.empty()) {
        st.p50_ms = v[(v.size() - 1) / 2];
        st.p99_ms = v[std::min(v.size() - 1, (size_t)std::ceil(0.99 * v.size()) - 1)];
        double sum = 0;
        for (double x : v) sum += x;
        st.mean_ms = sum / v.size();
        st.max_ms = v.back();
        st.wall_s = std::chrono::duration<double>(s->last - s->first).count();
        st.proofs_per_s = st.wall_s > 0 ? s->proofs / st.wall_s : 0;
    }
    st.mean_pack_rows = s->packs ? (double)s->pack_rows / s->packs : 0;
    st.rejected = s->rejected;
    st.nomem = s->nomem;
    st.cancelled = s->cancelled;
    st.mean_wait_ms = v.empty() ? 0 : s->sum_wait_ms / v.size();
    st.mean_enqueue_ms = s->packs ? s->sum_enqueue_ms / s->packs : 0;
    st.mean_run_ms = s->packs ? s->sum_run_ms / s->packs : 0;
    st.mean_msm_ms = s->packs ? s->sum_msm_ms / s->packs : 0;
    st.mean_launch_ms = s->launches ? s->sum_launch_ms / s->launches : 0;
    st.launches = s->launches;
    *out = st;
    return 0;
}

int fk20_server_reset_stats(fk20_server *s) {
    if (!s) return FK20_EINVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    s->lat_ms.clear();
    s->proofs = s->packs = s->pack_rows = s->rejected = s->nomem = s->cancelled = 0;
    s->sum_wait_ms = s->sum_enqueue_ms = s->sum_run_ms = s->sum_msm_ms = s->sum_launch_ms = 0;
    s->launches = 0;
    s->started = false;
    return 0;
}

int fk20_server_destroy(fk20_server *s) {
    if (!s) return FK20_EINVAL;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    server_free(s);
    delete s;
    return 0;
}

}  // extern "C"
