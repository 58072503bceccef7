// engine.cu -- host side of the B200 FK20 engine and its C ABI (include/fk20_b200.h).
//
// Owns
//   - the constant tables (GLV/NAF twiddle programs, Fr twiddles), computed
//     once on the host from the curve constants and uploaded to every kernel
//     module of every device used;
//   - contexts: fixed-base MSM tables per polynomial length, and workspaces;
//   - the launch sequence of every entry point.
// There is no CPU compute path: without a usable sm_100 device every entry
// point returns FK20_ENODEV or the CUDA error.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/fk20_b200.h"
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

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    int reserve(size_t need) {
        if (need <= bytes) return 0;
        if (p) {
            cudaDeviceSynchronize();  // the old buffer may still be in use by queued work
            cudaFree(p);
        }
        p = nullptr;
        bytes = 0;
        if (cudaMalloc(&p, need) != cudaSuccess) {
            cudaGetLastError();
            p = nullptr;
            return FK20_ENOMEM;
        }
        bytes = need;
        return 0;
    }
    void release() {
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
    unsigned long long fingerprint = 0;
};

}  // namespace

// Per-launch profiling: CUDA events on the launching stream around every
// pipeline kernel, with the algorithmic work of that launch (in 32x32->64-bit
// limb products: Fp product M_p = 300, Fr product M_r = 136, RCB addition
// 12 M_p, mixed addition 11 M_p, doubling 8 M_p).
struct Profiler {
    bool on = false;
    struct Rec {
        int kind;
        double products;
        cudaEvent_t a, b;
    };
    std::vector<Rec> pending;
    std::vector<cudaEvent_t> pool;
    double ms[FK20_NKINDS] = {0}, products[FK20_NKINDS] = {0};
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
    void begin(int kind, double prod, cudaStream_t st) {
        if (!on) return;
        Rec r{kind, prod, get(), get()};
        cudaEventRecord(r.a, st);
        pending.push_back(r);
    }
    void end(cudaStream_t st) {
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
            launches[r.kind] += 1;
            pool.push_back(r.a);
            pool.push_back(r.b);
        }
        pending.clear();
    }
    void reset() {
        collect();
        for (int k = 0; k < FK20_NKINDS; k++) ms[k] = products[k] = 0, launches[k] = 0;
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
    int fused_fft = 1;  // run the G1 FFT stages as one persistent launch
    std::mutex mu;
    Tables tab[3];  // log_m 7, 8, 9
    DevBuf S, D, D2, scratch, xext, offs, fp_dev;
    // persistent-launch state: per-position readiness, task counter, error flag
    DevBuf ready, sync;
    unsigned epoch = 0;
    int *err_host = nullptr;  // pinned copy of the device error flag
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

// ---- algorithmic work model (limb products) ----------------------------------
constexpr double MP = 300.0, MR = 136.0, ADD_P = 12 * MP, MADD_P = 11 * MP, DBL_P = 8 * MP;

double prog_products(int idx) {
    const HostConsts &hc = host_consts();
    if (hc.prog[idx][0] & 0x300u) return 0.0;
    return hc.prog_dbl[idx] * DBL_P + hc.prog_add[idx] * ADD_P + MP;  // + phi(P)
}

// one stage over `rows` rows: kind 0 DIF inverse, 1 DIT forward
double stage_products(int rows, int log_m, int s, int kind) {
    const int m = 1 << log_m;
    double per_row = 0;
    for (int b = 0; b < m / 2; b++) {
        int tix;
        if (kind == 0) {
            const int half = m >> (s + 1), j = b & (half - 1);
            tix = ((m - (j << s)) << (MAX_LOG_M - log_m)) & 511;
        } else {
            const int half = 1 << s, j = b & (half - 1);
            tix = (j << (log_m - 1 - s)) << (MAX_LOG_M - log_m);
        }
        per_row += 2 * ADD_P + (tix ? prog_products(tix) : 0.0);
    }
    return per_row * rows;
}

double fr_fft_products(int log_m) {  // nontrivial twiddle products of one Fr FFT-m
    const int m = 1 << log_m;
    return ((double)log_m * (m / 2) - (m - 1)) * MR;
}

// inverse DIF stages 0..L-2, middle (last inverse + zero upper half + first
// forward stage, optionally times 1/m), forward DIT stages 1..L-1
int run_hext_to_hfft(Profiler &pf, uint4 *D, int G, int rows, int log_m, int scale, cudaStream_t st) {
    const int m = 1 << log_m;
    for (int s = 0; s < log_m - 1; s++) {
        pf.begin(FK20_K_STAGE_INV, stage_products(rows, log_m, s, 0), st);
        launch_g1_stage(D, G, log_m, s, 0, st);
        pf.end(st);
        CKL();
    }
    pf.begin(FK20_K_MIDDLE, (double)rows * (m / 2) * (ADD_P + (scale ? prog_products(512 + log_m) : 0.0)), st);
    launch_g1_middle(D, G, log_m, scale, st);
    pf.end(st);
    CKL();
    for (int s = 1; s < log_m; s++) {
        pf.begin(FK20_K_STAGE_FWD, stage_products(rows, log_m, s, 1), st);
        launch_g1_stage(D, G, log_m, s, 1, st);
        pf.end(st);
        CKL();
    }
    return 0;
}

// the same sequence as one persistent launch (kernels_fft.cu k_g1_fused)
int run_hext_to_hfft_fused(fk20_ctx *ctx, uint4 *D, int G, int rows, int log_m, cudaStream_t st) {
    const int m = 1 << log_m;
    const size_t ready_bytes = (size_t)G * m * sizeof(unsigned);
    if (ctx->ready.bytes < ready_bytes) {
        CKR(ctx->ready.reserve(ready_bytes));
        CK(cudaMemsetAsync(ctx->ready.p, 0, ctx->ready.bytes, st));
        ctx->epoch = 0;
    }
    CKR(ctx->sync.reserve(256));
    if (++ctx->epoch >= (1u << 26)) {  // counters carry epoch * 64: restart before they wrap
        CK(cudaMemsetAsync(ctx->ready.p, 0, ctx->ready.bytes, st));
        ctx->epoch = 1;
    }
    unsigned *next = (unsigned *)ctx->sync.p;
    int *err = (int *)((char *)ctx->sync.p + 128);
    CK(cudaMemsetAsync(next, 0, sizeof(unsigned), st));
    CK(cudaMemsetAsync(err, 0, sizeof(int), st));
    double prod = 0;
    for (int s = 0; s < log_m - 1; s++) prod += stage_products(rows, log_m, s, 0) + stage_products(rows, log_m, s + 1, 1);
    prod += (double)rows * (m / 2) * ADD_P;
    ctx->prof.begin(FK20_K_FFT_FUSED, prod, st);
    launch_g1_fused(D, (unsigned *)ctx->ready.p, next, err, ctx->epoch, G, log_m, ctx->sms, st);
    ctx->prof.end(st);
    CKL();
    if (ctx->err_host) CK(cudaMemcpyAsync(ctx->err_host, err, sizeof(int), cudaMemcpyDeviceToHost, st));
    return 0;
}

// the inverse + forward transforms of the pipeline, fused or stage by stage
int run_pipeline_fft(fk20_ctx *ctx, uint4 *D, int G, int rows, int log_m, cudaStream_t st) {
    if (ctx->err_host && *ctx->err_host) return FK20_ETIMEOUT;  // a previous fused launch gave up
    if (ctx->fused_fft) return run_hext_to_hfft_fused(ctx, D, G, rows, log_m, st);
    return run_hext_to_hfft(ctx->prof, D, G, rows, log_m, 0, st);
}

int output_launch(Profiler &pf, uint64_t *dst, const uint4 *D, const size_t *row_off, int rows, int log_m,
                  int bitrev_out, cudaStream_t st) {
    pf.begin(FK20_K_OUTPUT, (double)rows * (1 << log_m) * 3 * MP, st);
    launch_tile_to_ref(dst, D, row_off, rows, log_m, bitrev_out, st);
    pf.end(st);
    CKL();
    return 0;
}

int build_tables(fk20_ctx *ctx, int log_m, const uint64_t *xext, cudaStream_t st) {
    Tables *T = tables_for(ctx, log_m);
    const int m = 1 << log_m;
    const int cb = ctx->window;
    const int W = (255 + cb - 1) / cb;
    const int E = 1 << (cb - 1);
    const int nbases = L_COLS * m;
    const size_t entries = (size_t)nbases * W * E;
    T->ready = false;
    T->table.release();
    CKR(T->table.reserve(entries * 6 * sizeof(uint4)));
    // slabs of bases keep the Z scratch near 1 GiB
    const size_t per_base_z = (size_t)W * E * table_z_bytes();
    int slab = (int)std::max<size_t>(1, (1ull << 30) / per_base_z);
    slab = std::min(slab, nbases);
    CKR(ctx->scratch.reserve((size_t)slab * per_base_z + (size_t)slab * W * table_window_base_bytes()));
    void *zs = ctx->scratch.p;
    void *wb = (char *)ctx->scratch.p + (size_t)slab * per_base_z;
    for (int b0 = 0; b0 < nbases; b0 += slab) {
        const int nb = std::min(slab, nbases - b0);
        launch_table_windows(wb, xext, b0, nb, W, cb, 512 + log_m, st);
        CKL();
        launch_table_fill((uint4 *)T->table.p, zs, wb, b0, nb, W, cb, st);
        CKL();
        launch_table_affine((uint4 *)T->table.p, zs, b0, nb, W, cb, st);
        CKL();
    }
    T->n = (unsigned)(m * L_COLS / 2);
    T->log_m = log_m;
    T->cb = cb;
    T->W = W;
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

int msm_launch(Profiler &pf, Tables *T, uint4 *D, const uint4 *S, int G, int rows, int times_m, cudaStream_t st) {
    MsmArgs a;
    a.D = D;
    a.S = S;
    a.table = (const uint4 *)T->table.p;
    a.G = G;
    a.log_m = T->log_m;
    a.rows = rows;
    a.cb = T->cb;
    a.W = T->W;
    a.times_m = times_m;
    const double prod = (double)rows * L_COLS * (1 << T->log_m) * T->W * MADD_P +
                        (times_m ? (double)rows * (1 << T->log_m) * T->log_m * DBL_P : 0.0);
    pf.begin(FK20_K_MSM, prod, st);
    launch_msm(a, st);
    pf.end(st);
    CKL();
    return 0;
}

// polynomial rows -> tiles of hext_fft (times 1/m unless times_m) in ctx->D
int pipeline_to_hext(fk20_ctx *ctx, Tables *T, const fr_t *poly, const size_t *row_off, unsigned rows, int times_m,
                     cudaStream_t st) {
    const int log_m = T->log_m, m = 1 << log_m;
    const int G = (int)((rows + 31) / 32);
    CKR(ctx->S.reserve(scal_bytes(G, m)));
    CKR(ctx->D.reserve(tile_bytes(G, m)));
    ctx->prof.begin(FK20_K_TC_FFT, (double)rows * L_COLS * fr_fft_products(log_m), st);
    launch_tc_fft((uint4 *)ctx->S.p, (const uint64_t *)poly, row_off, (int)T->n, log_m, rows, st);
    ctx->prof.end(st);
    CKL();
    CKR(msm_launch(ctx->prof, T, (uint4 *)ctx->D.p, (const uint4 *)ctx->S.p, G, (int)rows, times_m, st));
    return 0;
}

int check_call(const void *out, const void *in, unsigned rows) {
    if (!out || !in) return FK20_EINVAL;
    if (rows == 0 || rows > MAX_ROWS) return FK20_EINVAL;
    if (((uintptr_t)out | (uintptr_t)in) & 15) return FK20_EINVAL;
    return 0;
}

// ---- default context for the reference-signature entry points ---------------
std::mutex g_default_mu;
fk20_ctx *g_default[64];

int default_ctx(fk20_ctx **out) {
    int dev;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) { cudaGetLastError(); return FK20_ENODEV; }
    std::lock_guard<std::mutex> lk(g_default_mu);
    if (!g_default[dev]) CKR(fk20_ctx_create(&g_default[dev], dev, 0));
    *out = g_default[dev];
    return 0;
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

int fk20_ctx_create(fk20_ctx **out, int device, int window) {
    if (!out) return FK20_EINVAL;
    if (window == 0) window = 10;
    if (window < 8 || window > 13) return FK20_EINVAL;
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
        if (cudaMallocHost(&c->err_host, sizeof(int)) == cudaSuccess) *c->err_host = 0;
        else { cudaGetLastError(); c->err_host = nullptr; }
    }
    *out = c;
    return 0;
}

int fk20_ctx_set(fk20_ctx *ctx, int option, int value) {
    if (!ctx) return FK20_EINVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    switch (option) {
    case FK20_OPT_FUSED_FFT: ctx->fused_fft = value != 0; return 0;
    default: return FK20_EINVAL;
    }
}

int fk20_ctx_status(fk20_ctx *ctx) {
    if (!ctx) return FK20_EINVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    DeviceGuard dg(ctx->device);
    CK(cudaDeviceSynchronize());
    if (ctx->err_host && *ctx->err_host) {
        *ctx->err_host = 0;
        return FK20_ETIMEOUT;
    }
    return 0;
}

int fk20_ctx_destroy(fk20_ctx *ctx) {
    if (!ctx) return FK20_EINVAL;
    {
        DeviceGuard dg(ctx->device);
        cudaDeviceSynchronize();
        for (auto &t : ctx->tab) t.table.release();
        ctx->S.release();
        ctx->D.release();
        ctx->D2.release();
        ctx->scratch.release();
        ctx->xext.release();
        ctx->offs.release();
        ctx->fp_dev.release();
        ctx->ready.release();
        ctx->sync.release();
        if (ctx->err_host) cudaFreeHost(ctx->err_host);
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

int fk20_program_cost(int index, int *dbl, int *add) {
    if (index < 0 || index >= NPROG || !dbl || !add) return FK20_EINVAL;
    const HostConsts &hc = host_consts();
    *dbl = hc.prog_dbl[index];
    *add = hc.prog_add[index];
    return 0;
}

size_t fk20_ctx_device_bytes(const fk20_ctx *ctx) {
    if (!ctx) return 0;
    size_t b = ctx->S.bytes + ctx->D.bytes + ctx->D2.bytes + ctx->scratch.bytes + ctx->xext.bytes + ctx->offs.bytes;
    for (auto &t : ctx->tab) b += t.table.bytes;
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
    cudaStream_t st = S_(stream);
    const int G = (int)((rows + 31) / 32);
    CKR(pipeline_to_hext(ctx, T, polynomial, nullptr, rows, 0, st));
    CKR(run_pipeline_fft(ctx, (uint4 *)ctx->D.p, G, (int)rows, log_m, st));
    CKR(output_launch(ctx->prof, (uint64_t *)h_fft, (const uint4 *)ctx->D.p, nullptr, (int)rows, log_m, 0, st));
    return 0;
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
    cudaStream_t st = S_(stream);
    CKR(pipeline_to_hext(ctx, T, polynomial, nullptr, rows, 1, st));
    CKR(output_launch(ctx->prof, (uint64_t *)hext_fft, (const uint4 *)ctx->D.p, nullptr, (int)rows, log_m, 0, st));
    return 0;
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
    CKR(ctx->S.reserve(scal_bytes(G, m)));
    CKR(ctx->D.reserve(tile_bytes(G, m)));
    launch_ref_to_scalars((uint4 *)ctx->S.p, (const uint64_t *)tc_fft, (int)rows, log_m, st);
    CKL();
    CKR(msm_launch(ctx->prof, T, (uint4 *)ctx->D.p, (const uint4 *)ctx->S.p, G, (int)rows, 1, st));
    CKR(output_launch(ctx->prof, (uint64_t *)hext_fft, (const uint4 *)ctx->D.p, nullptr, (int)rows, log_m, 0, st));
    return 0;
}

int fk20_ctx_batch(fk20_ctx *ctx, g1p_t *h_fft, const fr_t *polys, unsigned count, const unsigned *n,
                   const size_t *poly_off, const size_t *out_off, void *stream) {
    if (!ctx || !h_fft || !polys || !n || !poly_off || !out_off || count == 0 || count > MAX_ROWS) return FK20_EINVAL;
    if (((uintptr_t)h_fft | (uintptr_t)polys) & 15) return FK20_EINVAL;
    for (unsigned j = 0; j < count; j++)
        if (log_m_for_n(n[j]) < 0) return FK20_EINVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    DeviceGuard dg(ctx->device);
    cudaStream_t st = S_(stream);
    // group instances by length; one stream-ordered pipeline per length
    std::vector<size_t> offs;
    struct Group { int log_m; size_t first; unsigned rows; };
    std::vector<Group> groups;
    for (int log_m = 9; log_m >= 7; log_m--) {
        const unsigned nn = (unsigned)(L_COLS << (log_m - 1));
        Group gr{log_m, offs.size(), 0};
        for (unsigned j = 0; j < count; j++)
            if (n[j] == nn) { offs.push_back(poly_off[j]); gr.rows++; }
        for (unsigned j = 0; j < count; j++)
            if (n[j] == nn) offs.push_back(out_off[j]);
        if (gr.rows) {
            if (!tables_for(ctx, log_m)->ready) return FK20_ENOSETUP;
            groups.push_back(gr);
        }
    }
    CKR(ctx->offs.reserve(offs.size() * sizeof(size_t)));
    CK(cudaMemcpyAsync(ctx->offs.p, offs.data(), offs.size() * sizeof(size_t), cudaMemcpyHostToDevice, st));
    const size_t *doffs = (const size_t *)ctx->offs.p;
    for (const Group &gr : groups) {
        Tables *T = tables_for(ctx, gr.log_m);
        const int G = (int)((gr.rows + 31) / 32);
        CKR(pipeline_to_hext(ctx, T, polys, doffs + gr.first, gr.rows, 0, st));
        CKR(run_pipeline_fft(ctx, (uint4 *)ctx->D.p, G, (int)gr.rows, gr.log_m, st));
        CKR(output_launch(ctx->prof, (uint64_t *)h_fft, (const uint4 *)ctx->D.p, doffs + gr.first + gr.rows,
                          (int)gr.rows, gr.log_m, 0, st));
    }
    // the host offset array must outlive the copy from pageable memory
    CK(cudaStreamSynchronize(st));
    return 0;
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
