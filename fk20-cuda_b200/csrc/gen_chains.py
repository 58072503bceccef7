#!/usr/bin/env python3
"""Writes chains.inc: the carry chains of the Fp (12 x 32-bit limbs) and Fr
(8 limbs) arithmetic in field.cuh, each chain ONE inline-PTX statement.

A chain of add.cc / addc.cc / mad.lo.cc / madc.hi.cc ... instructions passes
the carry flag CC.CF from one instruction to the next.  The flag is invisible
to the compiler, so a chain written as separate asm statements depends on
nothing being placed between them that also writes the flag.  Here every
chain starts with an instruction that does not read the flag and ends with
one whose flag output is not used, and lives entirely inside one asm
statement, so no code can come between its links.

The generated functions are specialisations for the two descriptors FpDesc
and FrDesc (field.cuh); the modulus enters as immediates ("n" operands) read
from the descriptor, so the constants have one source.  Host builds use the
portable stand-ins in field.cuh instead (ch_* there call these in
device code).

Run from this directory: python gen_chains.py > chains.inc"""

FIELDS = (("FpDesc", 12), ("FrDesc", 8))


def block(name, sig, lines, outs, ins, temps=()):
    """One device function whose body is a single asm statement."""
    body = []
    if temps:
        body.append('"{\\n\\t"')
        body.append('".reg .u32 %s;\\n\\t"' % ", ".join(temps))
    body += ['"%s;\\n\\t"' % l for l in lines]
    if temps:
        body.append('"}"')
    txt = "template <> FK_D %s %s<%s>(%s) {\n" % (sig[0], name, sig[1], sig[2])
    txt += sig[3]
    txt += "    asm volatile(" + "\n        ".join(body) + "\n"
    txt += "        : " + ", ".join(outs) + "\n"
    txt += "        : " + ", ".join(ins) + ");\n"
    txt += sig[4]
    txt += "}\n"
    return txt


def gen(desc, n):
    out = []
    half = n // 2

    # r = a + b (the carry out of the top word is dropped: callers keep sums < 2^(32n))
    outs = ['"=r"(r[%d])' % i for i in range(n)]
    ins = ['"r"(a[%d])' % i for i in range(n)] + ['"r"(b[%d])' % i for i in range(n)]
    A = lambda i: "%%%d" % (n + i)
    B = lambda i: "%%%d" % (2 * n + i)
    lines = ["add.cc.u32 %%0, %s, %s" % (A(0), B(0))]
    lines += ["addc.cc.u32 %%%d, %s, %s" % (i, A(i), B(i)) for i in range(1, n - 1)]
    lines += ["addc.u32 %%%d, %s, %s" % (n - 1, A(n - 1), B(n - 1))]
    out.append(block("ptx_add", ("void", desc, "uint32_t *r, const uint32_t *a, const uint32_t *b", "", ""),
                     lines, outs, ins))

    # r = a - b; returns all ones when a < b (a borrow out of the top word), else 0
    outs = ['"=r"(r[%d])' % i for i in range(n)] + ['"=r"(mask)']
    Ai = lambda i: "%%%d" % (n + 1 + i)
    Bi = lambda i: "%%%d" % (2 * n + 1 + i)
    lines = ["sub.cc.u32 %%0, %s, %s" % (Ai(0), Bi(0))]
    lines += ["subc.cc.u32 %%%d, %s, %s" % (i, Ai(i), Bi(i)) for i in range(1, n)]
    lines += ["subc.u32 %%%d, 0, 0" % n]
    out.append(block("ptx_sub", ("uint32_t", desc, "uint32_t *r, const uint32_t *a, const uint32_t *b",
                                "    uint32_t mask;\n", "    return mask;\n"), lines, outs, ins))

    # r = t - modulus; returns all ones when t < modulus
    ins = ['"r"(t[%d])' % i for i in range(n)] + ['"n"(%s::mod(%d))' % (desc, i) for i in range(n)]
    lines = ["sub.cc.u32 %%0, %s, %s" % (Ai(0), Bi(0))]
    lines += ["subc.cc.u32 %%%d, %s, %s" % (i, Ai(i), Bi(i)) for i in range(1, n)]
    lines += ["subc.u32 %%%d, 0, 0" % n]
    out.append(block("ptx_sub_mod", ("uint32_t", desc, "uint32_t *r, const uint32_t *t",
                                    "    uint32_t mask;\n", "    return mask;\n"), lines, outs, ins))

    # product row, even half: e[0..n-1] += a[j] * b for even j (lo word at j,
    # hi word at j + 1); e[n] = the carry out (its old value is not read)
    outs = ['"+r"(e[%d])' % i for i in range(n)] + ['"=r"(e[%d])' % n]
    ins = ['"r"(a[%d])' % (2 * k) for k in range(half)] + ['"r"(b)']
    a_ = lambda k: "%%%d" % (n + 1 + k)
    b_ = "%%%d" % (n + 1 + half)
    lines = []
    for k in range(half):
        lo, hi = 2 * k, 2 * k + 1
        lines.append("%s.u32 %%%d, %s, %s, %%%d" % ("mad.lo.cc" if k == 0 else "madc.lo.cc", lo, a_(k), b_, lo))
        lines.append("madc.hi.cc.u32 %%%d, %s, %s, %%%d" % (hi, a_(k), b_, hi))
    lines.append("addc.u32 %%%d, 0, 0" % n)
    out.append(block("ptx_row_even", ("void", desc, "uint32_t *e, const uint32_t *a, uint32_t b", "", ""),
                     lines, outs, ins))

    # product row, odd half: o[0] += c, then o[1..n] += a[j] * b for odd j
    # (lo word at j, hi word at j + 1); o[n] is overwritten (its old value is 0)
    outs = ['"+r"(o[%d])' % i for i in range(n)] + ['"=r"(o[%d])' % n]
    ins = ['"r"(a[%d])' % (2 * k + 1) for k in range(half)] + ['"r"(b)', '"r"(c)']
    c_ = "%%%d" % (n + 1 + half + 1)
    lines = ["add.cc.u32 %%0, %%0, %s" % c_]
    for k in range(half):
        lo, hi = 2 * k + 1, 2 * k + 2
        lines.append("madc.lo.cc.u32 %%%d, %s, %s, %%%d" % (lo, a_(k), b_, lo))
        if k < half - 1:
            lines.append("madc.hi.cc.u32 %%%d, %s, %s, %%%d" % (hi, a_(k), b_, hi))
        else:
            lines.append("madc.hi.u32 %%%d, %s, %s, 0" % (hi, a_(k), b_))
    out.append(block("ptx_row_odd", ("void", desc, "uint32_t *o, const uint32_t *a, uint32_t b, uint32_t c", "", ""),
                     lines, outs, ins))

    # reduction, even half: e[0..n-1] += m * mod[j] for even j; e[n] += carry
    outs = ['"+r"(e[%d])' % i for i in range(n + 1)]
    ins = ['"r"(m)'] + ['"n"(%s::mod(%d))' % (desc, 2 * k) for k in range(half)]
    m_ = "%%%d" % (n + 1)
    p_ = lambda k: "%%%d" % (n + 2 + k)
    lines = []
    for k in range(half):
        lo, hi = 2 * k, 2 * k + 1
        lines.append("%s.u32 %%%d, %s, %s, %%%d" % ("mad.lo.cc" if k == 0 else "madc.lo.cc", lo, m_, p_(k), lo))
        lines.append("madc.hi.cc.u32 %%%d, %s, %s, %%%d" % (hi, m_, p_(k), hi))
    lines.append("addc.u32 %%%d, %%%d, 0" % (n, n))
    out.append(block("ptx_red_even", ("void", desc, "uint32_t *e, uint32_t m", "", ""), lines, outs, ins))

    # reduction, odd half: o[1..n] += m * mod[j] for odd j (o[0] untouched)
    outs = ['"+r"(o[%d])' % i for i in range(1, n + 1)]
    ins = ['"r"(m)'] + ['"n"(%s::mod(%d))' % (desc, 2 * k + 1) for k in range(half)]
    m_ = "%%%d" % n
    q_ = lambda k: "%%%d" % (n + 1 + k)
    O = lambda w: "%%%d" % (w - 1)  # o[w] is operand w - 1
    lines = []
    for k in range(half):
        lo, hi = 2 * k + 1, 2 * k + 2
        lines.append("%s.u32 %s, %s, %s, %s" % ("mad.lo.cc" if k == 0 else "madc.lo.cc", O(lo), m_, q_(k), O(lo)))
        lines.append("%s.u32 %s, %s, %s, %s" % ("madc.hi.cc" if k < half - 1 else "madc.hi", O(hi), m_, q_(k), O(hi)))
    out.append(block("ptx_red_odd", ("void", desc, "uint32_t *o, uint32_t m", "", ""), lines, outs, ins))

    # squaring rows I = 1 .. n-1 (row 0 is plain products): e[j0..n-1] += v[j] * b
    # for even j >= I (lo word at j, hi word at j + 1), e[n] = the carry out;
    # o[j0..n] += v[j] * b for odd j >= I, o[n] written (its old value is 0)
    for I in range(1, n):
        for par, acc in ((0, "e"), (1, "o")):
            js = [j for j in range(I, n) if j % 2 == par]
            name = "ptx_sqrow_even" if par == 0 else "ptx_sqrow_odd"
            sig = ("void", "%s, %d" % (desc, I), "uint32_t *%s, const uint32_t *v, uint32_t b" % acc, "", "")
            if not js:
                out.append("template <> FK_D void %s<%s, %d>(uint32_t *, const uint32_t *, uint32_t) {}\n" % (name, desc, I))
                continue
            j0 = js[0]
            top = n if par == 0 else n + 1  # words j0 .. top - 1 are read and written
            words = list(range(j0, top))
            outs = []
            for w in words:
                last_even = par == 0 and w == n
                outs.append('"%s"(%s[%d])' % ("=r" if (w == n) else "+r", acc, w))
            if par == 0:
                outs.append('"=r"(%s[%d])' % (acc, n))
            op = {w: "%%%d" % k for k, w in enumerate(words + ([n] if par == 0 else []))}
            base = len(outs)
            ins = ['"r"(v[%d])' % j for j in js] + ['"r"(b)']
            vj = {j: "%%%d" % (base + k) for k, j in enumerate(js)}
            b_ = "%%%d" % (base + len(js))
            lines = []
            for k, j in enumerate(js):
                lo, hi = j, j + 1
                lines.append("%s.u32 %s, %s, %s, %s" % ("mad.lo.cc" if k == 0 else "madc.lo.cc", op[lo], vj[j], b_, op[lo]))
                if hi == n and par == 1:
                    lines.append("madc.hi.u32 %s, %s, %s, 0" % (op[hi], vj[j], b_))
                else:
                    lines.append("madc.hi.cc.u32 %s, %s, %s, %s" % (op[hi], vj[j], b_, op[hi]))
            if par == 0:
                lines.append("addc.u32 %s, 0, 0" % op[n])
            out.append(block(name, sig, lines, outs, ins))

    # t = (e + o + c) >> 32 over n + 1 words, c the pending word-0 carry (0 or 1)
    outs = ['"=r"(t[%d])' % i for i in range(n)]
    ins = ['"r"(e[%d])' % i for i in range(n + 1)] + ['"r"(o[%d])' % i for i in range(n + 1)] + ['"r"(c)']
    E = lambda i: "%%%d" % (n + i)
    Oo = lambda i: "%%%d" % (2 * n + 1 + i)
    c_ = "%%%d" % (3 * n + 2)
    lines = ["add.cc.u32 x, %s, -1" % c_, "addc.cc.u32 x, %s, %s" % (E(0), Oo(0))]
    lines += ["addc.cc.u32 %%%d, %s, %s" % (k - 1, E(k), Oo(k)) for k in range(1, n)]
    lines += ["addc.u32 %%%d, %s, %s" % (n - 1, E(n), Oo(n))]
    out.append(block("ptx_final_c", ("void", desc, "uint32_t *t, const uint32_t *e, const uint32_t *o, uint32_t c", "", ""),
                     lines, outs, ins, temps=("x",)))

    # t = (e + o) >> 32 over n + 1 words
    outs = ['"=r"(t[%d])' % i for i in range(n)]
    ins = ['"r"(e[%d])' % i for i in range(n + 1)] + ['"r"(o[%d])' % i for i in range(n + 1)]
    E = lambda i: "%%%d" % (n + i)
    Oo = lambda i: "%%%d" % (2 * n + 1 + i)
    lines = ["add.cc.u32 x, %s, %s" % (E(0), Oo(0))]
    lines += ["addc.cc.u32 %%%d, %s, %s" % (k - 1, E(k), Oo(k)) for k in range(1, n)]
    lines += ["addc.u32 %%%d, %s, %s" % (n - 1, E(n), Oo(n))]
    out.append(block("ptx_final", ("void", desc, "uint32_t *t, const uint32_t *e, const uint32_t *o", "", ""),
                     lines, outs, ins, temps=("x",)))
    return out


def main():
    print("// chains.inc -- written by gen_chains.py (run it to regenerate; do not edit).")
    print("// One asm statement per carry chain of the Fp and Fr arithmetic (field.cuh).")
    print("// clang-format off")
    for desc, n in FIELDS:
        print("\n// ---------------------------------------------------------------- %s (%d limbs)\n" % (desc, n))
        for f in gen(desc, n):
            print(f)
    # word-0 carry of the Montgomery loop, shared by both fields
    print("// the carry out of e0 + o0 (0 or 1)")
    print("FK_D uint32_t ptx_carry0(uint32_t e0, uint32_t o0) {")
    print("    uint32_t c;")
    print('    asm volatile("{\\n\\t"')
    print('        ".reg .u32 x;\\n\\t"')
    print('        "add.cc.u32 x, %1, %2;\\n\\t"')
    print('        "addc.u32 %0, 0, 0;\\n\\t"')
    print('        "}"')
    print('        : "=r"(c)')
    print('        : "r"(e0), "r"(o0));')
    print("    return c;")
    print("}")
    # carry out of e0 + o0 + c (c = 0 or 1): the carry flag is set to c first
    print("// the carry out of e0 + o0 + c, c = 0 or 1")
    print("FK_D uint32_t ptx_carry3(uint32_t e0, uint32_t o0, uint32_t c) {")
    print("    uint32_t r;")
    print('    asm volatile("{\\n\\t"')
    print('        ".reg .u32 x;\\n\\t"')
    print('        "add.cc.u32 x, %3, -1;\\n\\t"')
    print('        "addc.cc.u32 x, %1, %2;\\n\\t"')
    print('        "addc.u32 %0, 0, 0;\\n\\t"')
    print('        "}"')
    print('        : "=r"(r)')
    print('        : "r"(e0), "r"(o0), "r"(c));')
    print("    return r;")
    print("}")
    print("// clang-format on")


if __name__ == "__main__":
    main()
