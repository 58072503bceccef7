// Test probe of include/fk20_device.cuh: kernels that apply the reference-named
// device functions over arrays, behind plain C entry points (tests only).
#include "fk20_device.cuh"

__global__ void k_fp(int op, fp_t *z, const fp_t *x, const fp_t *y, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    fp_t r;
    switch (op) {
    case 0: fp_mul(r, x[i], y[i]); break;
    case 1: fp_sqr(r, x[i]); break;
    case 2: fp_add(r, x[i], y[i]); break;
    case 3: fp_sub(r, x[i], y[i]); break;
    case 4: fp_neg(r, x[i]); break;
    case 5: fp_inv(r, x[i]); break;
    case 6: fp_x3(r, x[i]); break;
    case 7: fp_x12(r, x[i]); break;
    case 8: fp_mma(r, x[i], y[i], y[i], y[i]); break;  // x y + y^2
    case 9: fp_cpy(r, x[i]); fp_reduce6(r); break;
    default: fp_zero(r); r[0] = fp_eq(x[i], y[i]); break;
    }
    fp_cpy(z[i], r);
}

__global__ void k_fr(int op, fr_t *z, const fr_t *x, const fr_t *y, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    fr_t r, t;
    fr_cpy(r, x[i]);
    switch (op) {
    case 0: fr_mul(r, y[i]); break;
    case 1: fr_sqr(r); break;
    case 2: fr_add(r, y[i]); break;
    case 3: fr_sub(r, y[i]); break;
    case 4: fr_neg(r); break;
    case 5: fr_inv(r); break;
    case 6: fr_x3(r); break;
    case 7: fr_cpy(t, y[i]); fr_addsub(r, t); break;  // r = x + y
    default: fr_reduce4(r); break;
    }
    fr_cpy(z[i], r);
}

__global__ void k_g1(int op, g1p_t *z, const g1p_t *x, const g1p_t *y, const fr_t *s, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    g1p_t p, q;
    g1p_cpy(p, x[i]);
    g1p_cpy(q, y[i]);
    g1a_t a;
    switch (op) {
    case 0: g1p_add(p, q); break;
    case 1: g1p_dbl(p); break;
    case 2: g1p_sub(p, q); break;
    case 3: g1p_neg(p); break;
    case 4: g1p_mul(p, s[i]); break;
    case 5: g1p_addsub(p, q); g1p_add(p, q); break;  // (x + y) + (x - y) = 2x
    case 6: g1a_fromG1p(a, q); g1p_add(p, a); break;  // x + affine(y)
    case 7: g1p_inf(p); p.x[0] = g1p_eq(x[i], y[i]); p.y[0] = g1p_isPoint(x[i]); p.z[0] = g1p_isInf(x[i]); break;
    default: g1a_fromG1p(a, p); g1p_fromG1a(p, a); break;  // affine round trip
    }
    g1p_cpy(z[i], p);
}

extern "C" int devapi_fp(int op, void *z, const void *x, const void *y, int n) {
    k_fp<<<(n + 127) / 128, 128>>>(op, (fp_t *)z, (const fp_t *)x, (const fp_t *)y, n);
    return (int)cudaDeviceSynchronize();
}
extern "C" int devapi_fr(int op, void *z, const void *x, const void *y, int n) {
    k_fr<<<(n + 127) / 128, 128>>>(op, (fr_t *)z, (const fr_t *)x, (const fr_t *)y, n);
    return (int)cudaDeviceSynchronize();
}
extern "C" int devapi_g1(int op, void *z, const void *x, const void *y, const void *s, int n) {
    k_g1<<<(n + 63) / 64, 64>>>(op, (g1p_t *)z, (const g1p_t *)x, (const g1p_t *)y, (const fr_t *)s, n);
    return (int)cudaDeviceSynchronize();
}

// Throughput of a dependent chain of standard-form products, `iters` per
// element: form 0 is fp_mul of the device API (two Montgomery products);
// form 1 converts both operands in, multiplies and converts back (four),
// the wrapper the API's cost is compared against.
__device__ __forceinline__ void fp_mul_convert(fp_t &z, const fp_t &x, const fp_t &y) {
    using namespace fk20_device_detail;
    fk::Fp a, b, t;
    load_words(t, x);
    fk::f_to_mont(a, t);
    load_words(t, y);
    fk::f_to_mont(b, t);
    fk::f_mul(a, a, b);
    plain(z, a);
}
__global__ void k_fp_rate(int form, fp_t *x, const fp_t *y, int n, int iters) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    fp_t a, b;
    fp_cpy(a, x[i]);
    fp_cpy(b, y[i]);
    if (form == 0)
        for (int k = 0; k < iters; k++) fp_mul(a, a, b);
    else
        for (int k = 0; k < iters; k++) fp_mul_convert(a, a, b);
    fp_cpy(x[i], a);
}
extern "C" int devapi_fp_rate(int form, void *x, const void *y, int n, int iters, float *ms) {
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    k_fp_rate<<<(n + 127) / 128, 128>>>(form, (fp_t *)x, (const fp_t *)y, n, 1);  // warm-up
    cudaEventRecord(e0);
    k_fp_rate<<<(n + 127) / 128, 128>>>(form, (fp_t *)x, (const fp_t *)y, n, iters);
    cudaEventRecord(e1);
    const int rc = (int)cudaEventSynchronize(e1);
    cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc ? rc : (int)cudaGetLastError();
}
