// Host build of the engine's field and curve code (csrc/field.cuh, g1.cuh)
// with the carry flag emulated in C -- CPU unit tests only.  Lets the limb
// schedules, reduction bounds and curve formulas be checked against the
// oracle without a GPU.  Standard-form uint64 I/O, reference layouts.
#include <cstring>
#include "field.cuh"
#include "g1.cuh"
#include "glv.cuh"

using namespace fk;

template <class F>
static void load(Elem<F> &e, const uint64_t *x) {
    for (int i = 0; i < F::N / 2; i++) { e.w[2 * i] = (uint32_t)x[i]; e.w[2 * i + 1] = (uint32_t)(x[i] >> 32); }
}
template <class F>
static void store(uint64_t *x, const Elem<F> &e) {
    for (int i = 0; i < F::N / 2; i++) x[i] = (uint64_t)e.w[2 * i] | ((uint64_t)e.w[2 * i + 1] << 32);
}

template <class F>
static int field_op(int op, uint64_t *out, const uint64_t *a, const uint64_t *b, long count) {
    const int L = F::N / 2;
    for (long i = 0; i < count; i++) {
        Elem<F> x, y, z, t;
        load(t, a + L * i);
        f_to_mont(x, t);
        if (b) { load(t, b + L * i); f_to_mont(y, t); } else { f_set_zero(y); }
        switch (op) {
        case 0: f_mul(z, x, y); break;
        case 1: f_sqr(z, x); break;
        case 2: f_add(z, x, y); break;
        case 3: f_sub(z, x, y); break;
        case 4: f_neg(z, x); break;
        case 5: f_inv(z, x); break;
        case 6: z = x; break;
        case 7: f_dbl(z, x); break;
        case 11: f_mul12(z, x); break;
        default: return -1;
        }
        f_from_mont(t, z);
        store(out + L * i, t);
    }
    return 0;
}

static void g1_load(G1P &p, const uint64_t *g) {
    Fp t;
    load(t, g); f_to_mont(p.x, t);
    load(t, g + 6); f_to_mont(p.y, t);
    load(t, g + 12); f_to_mont(p.z, t);
}
static void g1_store(uint64_t *g, const G1P &p) {
    Fp t;
    f_from_mont(t, p.x); store(g, t);
    f_from_mont(t, p.y); store(g + 6, t);
    f_from_mont(t, p.z); store(g + 12, t);
}

extern "C" {
int emul_fp_op(int op, uint64_t *out, const uint64_t *a, const uint64_t *b, long count) { return field_op<FpDesc>(op, out, a, b, count); }
int emul_fr_op(int op, uint64_t *out, const uint64_t *a, const uint64_t *b, long count) { return field_op<FrDesc>(op, out, a, b, count); }

// op: 0 add, 1 dbl, 2 madd (b affine: x,y of 12 limbs), 3 phi, 4 neg
int emul_g1_op(int op, uint64_t *out, const uint64_t *a, const uint64_t *b, long count) {
    for (long i = 0; i < count; i++) {
        G1P p, q, r;
        g1_load(p, a + 18 * i);
        switch (op) {
        case 0: g1_load(q, b + 18 * i); g1_add(r, p, q); break;
        case 1: g1_dbl(r, p); break;
        case 2: { Fp qx, qy, t; load(t, b + 12 * i); f_to_mont(qx, t); load(t, b + 12 * i + 6); f_to_mont(qy, t); g1_madd(r, p, qx, qy); } break;
        case 3: g1_phi(r, p); break;
        case 4: g1_neg(r, p); break;
        default: return -1;
        }
        g1_store(out + 18 * i, r);
    }
    return 0;
}
}

#include "scalar_prog.cuh"
extern "C" {
// [k] P through a GLV/NAF program built for k (standard form, 4 x u64)
int emul_g1_mul_prog(uint64_t *out, const uint64_t *pts, const uint64_t *k, long count, int *dbl, int *add) {
    uint32_t prog[PROG_WORDS];
    host::make_program(prog, k);
    host::program_cost(prog, dbl, add);
    for (long i = 0; i < count; i++) {
        G1P p, r;
        g1_load(p, pts + 18 * i);
        g1_mul_prog(r, p, prog);
        g1_store(out + 18 * i, r);
    }
    return 0;
}
}

extern "C" {
// the program words host::make_program builds for k (standard form, 4 x u64)
int emul_make_program(uint32_t *prog, const uint64_t *k) {
    host::make_program(prog, k);
    return PROG_WORDS;
}
}

#include "fused_plan.cuh"
extern "C" {
// The persistent G1 FFT's task schedule for nseg segments (G[k] row groups,
// FFT size 2^log_m[k]): writes each task's (seg, stage, g, i0, i1, tix, kind)
// as 7 ints and returns the task count (-1 if it exceeds cap).
// a launch whose segments run only the stages [s_lo, s_hi) (s_hi = 0: all)
long emul_fused_schedule_w(int nseg, const int *G, const int *log_m, const int *s_lo, const int *s_hi, int *out,
                           long cap) {
    FusedBlocks b{};
    b.nseg = nseg;
    for (int k = 0; k < nseg; k++) {
        b.G[k] = G[k], b.log_m[k] = log_m[k];
        b.s_lo[k] = (unsigned char)s_lo[k], b.s_hi[k] = (unsigned char)s_hi[k];
    }
    const unsigned total = fused_blocks_build(b);
    if ((long)total > cap) return -1;
    for (unsigned t = 0; t < total; t++) {
        FusedTask f;
        fused_task_decode(f, b, t);
        int *o = out + 7 * (size_t)t;
        o[0] = f.seg; o[1] = f.S; o[2] = f.g; o[3] = f.i0; o[4] = f.i1; o[5] = f.tix; o[6] = f.kind;
    }
    return (long)total;
}

long emul_fused_schedule(int nseg, const int *G, const int *log_m, int *out, long cap) {
    FusedBlocks b{};
    b.nseg = nseg;
    for (int k = 0; k < nseg; k++) b.G[k] = G[k], b.log_m[k] = log_m[k];
    const unsigned total = fused_blocks_build(b);
    if ((long)total > cap) return -1;
    for (unsigned t = 0; t < total; t++) {
        FusedTask f;
        fused_task_decode(f, b, t);
        int *o = out + 7 * (size_t)t;
        o[0] = f.seg; o[1] = f.S; o[2] = f.g; o[3] = f.i0; o[4] = f.i1; o[5] = f.tix; o[6] = f.kind;
    }
    return (long)total;
}
}

extern "C" {
// GLV split of count scalars (4 x u64 each, s < 2^255): out[2 i] = s mod lambda,
// out[2 i + 1] = s div lambda (2 x u64 each, the upper two words zero)
int emul_glv_split(uint64_t *out, const uint64_t *s, long count) {
    for (long i = 0; i < count; i++) {
        uint32_t w[8], a[4], b[4];
        for (int k = 0; k < 4; k++) { w[2 * k] = (uint32_t)s[4 * i + k]; w[2 * k + 1] = (uint32_t)(s[4 * i + k] >> 32); }
        glv_split(a, b, w);
        for (int k = 0; k < 2; k++) {
            out[8 * i + k] = (uint64_t)a[2 * k] | ((uint64_t)a[2 * k + 1] << 32);
            out[8 * i + 4 + k] = (uint64_t)b[2 * k] | ((uint64_t)b[2 * k + 1] << 32);
        }
        out[8 * i + 2] = out[8 * i + 3] = out[8 * i + 6] = out[8 * i + 7] = 0;
    }
    return 0;
}
}
