// ref_shim.cu -- C entry points over the reference's own CUDA library
// (lCardosoSantos/FK20-CUDA, compiled unmodified from its sources for sm_100a
// by oracle/ref/Makefile).  TEST INFRASTRUCTURE: used only to pin the oracle
// and the engine to the reference's actual outputs, and to time the
// reference kernels on the same GPU.  Symbol names differ from the engine's
// (ref_*), and the library is loaded on its own (RTLD_LOCAL).
#include <cuda_runtime.h>
#include "fk20.cuh"

extern "C" {

// the reference's host pipeline, fk20_poly2h_fft.cu:47-78 (rows <= 512)
int ref_fk20_poly2h_fft(g1p_t *h_fft, const fr_t *polynomial, const g1p_t *xext_fft, unsigned rows) {
    fk20_poly2h_fft(h_fft, polynomial, xext_fft, rows);
    return (int)cudaDeviceSynchronize();
}

// the same six launches, keeping every intermediate (fk20_poly2h_fft.cu:57-77)
int ref_fk20_stages(const fr_t *polynomial, const g1p_t *xext_fft, unsigned rows, fr_t *tc, fr_t *tc_fft,
                    g1p_t *hext_fft, g1p_t *h, g1p_t *h_fft) {
    cudaError_t err;
    err = cudaFuncSetAttribute(fr_fft_wrapper, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fr_sharedmem);
    if (err != cudaSuccess) return (int)err;
    err = cudaFuncSetAttribute(g1p_fft_wrapper, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)g1p_sharedmem);
    if (err != cudaSuccess) return (int)err;
    err = cudaFuncSetAttribute(g1p_ift_wrapper, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)g1p_sharedmem);
    if (err != cudaSuccess) return (int)err;
    fk20_poly2toeplitz_coefficients<<<rows, 256>>>(tc, polynomial);
    cudaMemcpy(tc_fft, tc, sizeof(fr_t) * 8192 * (size_t)rows, cudaMemcpyDeviceToDevice);
    fr_fft_wrapper<<<rows * 16, 256, fr_sharedmem>>>(tc_fft, tc_fft);
    fk20_msm<<<rows, 256>>>(hext_fft, tc_fft, xext_fft);
    g1p_ift_wrapper<<<rows, 256, g1p_sharedmem>>>(h, hext_fft);
    fk20_hext2h<<<rows, 256>>>(h);
    g1p_fft_wrapper<<<rows, 256, g1p_sharedmem>>>(h_fft, h);
    return (int)cudaDeviceSynchronize();
}

// timing helper: the reference pipeline with CUDA events around it (ms)
int ref_fk20_time(g1p_t *h_fft, const fr_t *polynomial, const g1p_t *xext_fft, unsigned rows, float *ms) {
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, 0);
    fk20_poly2h_fft(h_fft, polynomial, xext_fft, rows);
    cudaEventRecord(b, 0);
    cudaError_t err = cudaEventSynchronize(b);
    cudaEventElapsedTime(ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return (int)err;
}

}
