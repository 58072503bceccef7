// fk20_prove -- C++ host program over the C ABI of libfk20b200.so: proves a
// file of polynomials against a file of setup points and writes the proofs.
//
//   fk20_prove <n> <rows> <setup.bin> <poly.bin> <out.bin> [--da] [--window W]
//
//   setup.bin  n g1p_t setup points [s^i]G1, i < n (the reference's setup[0],
//              FK20Py/kzg_proofs.py:22-30), 144 bytes each, standard form
//   poly.bin   rows x n fr_t coefficients, 32 bytes each
//   out.bin    rows x 2n/16 g1p_t proofs h_fft (fk20_poly2h_fft's output), or
//              with --da rows x 2n/16 48-byte compressed proofs in
//              bit-reversed order (data_availabilty_using_fk20_multi,
//              FK20Py/fk20_multi.py:107-118)
//
// It is the call sequence a C++ caller of the reference switches to:
// fk20_ctx_create, fk20_ctx_load_setup (setup -> xext_fft -> tables on the
// GPU), fk20_ctx_poly2h_fft / fk20_ctx_poly2proofs, fk20_ctx_destroy.  Exit
// status 0 on success, 1 with a message on any error.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "fk20_b200.h"

namespace {

int fail(const std::string &what, int code) {
    std::fprintf(stderr, "fk20_prove: %s failed (%d)\n", what.c_str(), code);
    return 1;
}

bool read_file(const char *path, std::vector<unsigned char> &buf, size_t bytes) {
    FILE *f = std::fopen(path, "rb");
    if (!f) return false;
    buf.resize(bytes);
    const size_t got = std::fread(buf.data(), 1, bytes, f);
    std::fclose(f);
    return got == bytes;
}

struct Device {  // cudaMalloc'd buffer released on scope exit
    void *p = nullptr;
    ~Device() {
        if (p) cudaFree(p);
    }
};

}  // namespace

int main(int argc, char **argv) {
    if (argc < 6) {
        std::fprintf(stderr, "usage: fk20_prove <n> <rows> <setup.bin> <poly.bin> <out.bin> [--da] [--window W]\n");
        return 1;
    }
    const unsigned n = (unsigned)std::strtoul(argv[1], nullptr, 10);
    const unsigned rows = (unsigned)std::strtoul(argv[2], nullptr, 10);
    bool da = false;
    int window = 10;
    for (int i = 6; i < argc; i++) {
        if (!std::strcmp(argv[i], "--da")) da = true;
        else if (!std::strcmp(argv[i], "--window") && i + 1 < argc) window = std::atoi(argv[++i]);
    }
    if ((n != 1024 && n != 2048 && n != 4096) || rows == 0) {
        std::fprintf(stderr, "fk20_prove: n must be 1024, 2048 or 4096 and rows > 0\n");
        return 1;
    }
    const size_t m = 2 * (size_t)n / 16;
    const size_t setup_b = (size_t)n * sizeof(g1p_t), poly_b = (size_t)rows * n * sizeof(fr_t);
    const size_t out_b = (size_t)rows * m * (da ? 48 : sizeof(g1p_t));
    std::vector<unsigned char> setup, poly, out(out_b);
    if (!read_file(argv[3], setup, setup_b)) return fail(std::string("reading ") + argv[3], 0);
    if (!read_file(argv[4], poly, poly_b)) return fail(std::string("reading ") + argv[4], 0);

    Device dsetup, dpoly, dout;
    cudaError_t ce;
    if ((ce = cudaMalloc(&dsetup.p, setup_b)) || (ce = cudaMalloc(&dpoly.p, poly_b)) ||
        (ce = cudaMalloc(&dout.p, out_b)))
        return fail("cudaMalloc", (int)ce);
    if ((ce = cudaMemcpy(dsetup.p, setup.data(), setup_b, cudaMemcpyHostToDevice)) ||
        (ce = cudaMemcpy(dpoly.p, poly.data(), poly_b, cudaMemcpyHostToDevice)))
        return fail("cudaMemcpy to the device", (int)ce);

    fk20_ctx *ctx = nullptr;
    int rc = fk20_ctx_create(&ctx, 0, window);
    if (rc) return fail("fk20_ctx_create", rc);
    rc = fk20_ctx_load_setup(ctx, n, (const g1p_t *)dsetup.p, nullptr);
    if (!rc) {
        if (da) rc = fk20_ctx_poly2proofs(ctx, (uint8_t *)dout.p, (const fr_t *)dpoly.p, rows, n, nullptr);
        else rc = fk20_ctx_poly2h_fft(ctx, (g1p_t *)dout.p, (const fr_t *)dpoly.p, rows, n, nullptr);
    }
    if (!rc) rc = (int)cudaDeviceSynchronize();
    const int rc_destroy = fk20_ctx_destroy(ctx);
    if (rc) return fail(da ? "proving (fk20_ctx_poly2proofs)" : "proving (fk20_ctx_poly2h_fft)", rc);
    if (rc_destroy) return fail("fk20_ctx_destroy", rc_destroy);
    if ((ce = cudaMemcpy(out.data(), dout.p, out_b, cudaMemcpyDeviceToHost))) return fail("cudaMemcpy to the host", (int)ce);

    FILE *f = std::fopen(argv[5], "wb");
    if (!f || std::fwrite(out.data(), 1, out_b, f) != out_b) {
        if (f) std::fclose(f);
        return fail(std::string("writing ") + argv[5], 0);
    }
    std::fclose(f);
    return 0;
}
