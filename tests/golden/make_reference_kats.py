"""Extract the reference's known-answer vectors into tests/golden/reference_kats.json.

Reads (as text) the KAT tables of lCardosoSantos/FK20-CUDA:
  fptest_kat.cu:18-718   FpTestKAT   (fp_cpy, fp_reduce6, fp_eq/neq, fp_neg, fp_x2, fp_x3,
                                       fp_add, fp_sub, fp_sqr, fp_mul, fp_inv, Mandelbrot)
  frtest_kat.cu:15-650   FrTestKAT   (fr_cpy, fr_reduce4, fr_eq/neq, fr_neg, fr_x2, fr_x3,
                                       fr_add, fr_sub, fr_sqr, fr_mul, fr_inv)
  g1test_kat.cu:10-60    g1p_x2, g1p_x3, g1p_x24, g1p_x25, g1p_wG, g1p_w8G
  fr_fft_testvector.cu   q[512] -> a[512] = fft(q)
  fr_roots.cu:17-533     fr_roots[515]

Each section's operation is mapped by hand from the kernel body that consumes
the table (the op name and which arrays are inputs / expected output); the
loop bound of the consuming loop is honoured.  Run this where the reference
tree is mounted:  python tests/golden/make_reference_kats.py [REF_DIR]
"""
import json
import os
import re
import sys

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("FK20_REFERENCE", "/root/reference")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_kats.json")

ROW = re.compile(r"\{\s*((?:0x[0-9a-fA-F]+\s*,\s*)*0x[0-9a-fA-F]+)\s*,?\s*\}")
ARR = re.compile(r"\b([a-z])\[\](?:\[\d\])?\s*=\s*\{")


def limbs_to_hex(limbs):
    v = 0
    for i, x in enumerate(limbs):
        v |= int(x, 16) << (64 * i)
    return hex(v)


def parse_arrays(body):
    """name -> list of hex ints, for every `x[] = { {..}, {..} }` in body."""
    arrays = {}
    for m in ARR.finditer(body):
        name = m.group(1)
        # find the matching closing brace of the outer initialiser
        depth, i = 0, m.end() - 1
        while True:
            if body[i] == "{":
                depth += 1
            elif body[i] == "}":
                depth -= 1
                if depth == 0:
                    break
            i += 1
        inner = body[m.end():i]
        rows = [limbs_to_hex([t.strip() for t in r.group(1).split(",")]) for r in ROW.finditer(inner)]
        arrays[name] = rows
    return arrays


def sections(text):
    """Split a KAT kernel body at the `    // name` section comments."""
    parts = re.split(r"\n    // ([^\n]+)\n", text)
    out = {}
    for k in range(1, len(parts), 2):
        out[parts[k].strip()] = parts[k + 1]
    return out


def loop_bound(body):
    m = re.search(r"for \(int i=0; (?:pass && )?\(?i<(\d+)\)?;", body)
    return int(m.group(1)) if m else None


def field_kats(path, prefix):
    text = open(path).read()
    secs = sections(text)
    kats = []
    unary = {"neg": "neg", "x2": "x2", "x3": "x3", "sqr": "sqr", "inv": "inv"}
    for name, body in secs.items():
        arrs = parse_arrays(body)
        nb = loop_bound(body)
        key = name.replace(prefix + "_", "")
        if key == "cpy":
            kats.append({"op": "cpy", "q": arrs["q"][:nb], "a": arrs["a"][:nb], "exact": True})
        elif key in ("reduce6", "reduce4"):
            kats.append({"op": "reduce", "q": arrs["q"][:nb], "a": arrs["a"][:nb], "exact": True})
        elif key.startswith("eq"):
            kats.append({"op": "eq", "t": arrs["t"], "u": arrs["u"]})
        elif key in unary:
            # fr_inv compares limbs exactly (frtest_kat.cu:600-606); the rest via neq
            kats.append({"op": unary[key], "q": arrs["q"][:nb], "a": arrs["a"][:nb],
                         "exact": prefix == "fr" and key == "inv"})
        elif key in ("add", "sub", "mul"):
            kats.append({"op": key, "x": arrs["x"][:nb], "y": arrs["y"][:nb], "a": arrs["a"][:nb]})
        elif key.startswith("Mandelbrot"):
            kats.append({"op": "mandelbrot", "iterations": 10000, "q": arrs["q"], "a": arrs["a"]})
        else:
            raise SystemExit(f"unmapped section {name!r} in {path}")
    return kats


def g1_kats(path):
    text = open(path).read()
    pts = {}
    for m in re.finditer(r"(g1p_\w+) = \{(.*?)\n    \}", text, re.S):
        rows = [limbs_to_hex([t.strip() for t in r.group(1).split(",")]) for r in ROW.finditer(m.group(2))]
        pts[m.group(1)] = rows
    # g1p_x0 is the ANYINF infinity (0, (1,2,3,4,5,6), 0), g1test_kat.cu:11-18
    return {k: v for k, v in pts.items()}


def fft_vector(path):
    text = open(path).read()
    q = text[text.index("q[512]"):text.index("a[512]")]
    a = text[text.index("a[512]"):]
    qs = [limbs_to_hex([t.strip() for t in r.group(1).split(",")]) for r in ROW.finditer(q)]
    as_ = [limbs_to_hex([t.strip() for t in r.group(1).split(",")]) for r in ROW.finditer(a)]
    assert len(qs) == 512 and len(as_) == 512, (len(qs), len(as_))
    return {"q": qs, "a": as_}


def roots(path):
    text = open(path).read()
    body = text[text.index("fr_roots[515]"):text.index("fr_roots_host")]
    rs = [limbs_to_hex([t.strip() for t in r.group(1).split(",")]) for r in ROW.finditer(body)]
    assert len(rs) == 515, len(rs)
    return rs


def main():
    data = {
        "source": "lCardosoSantos/FK20-CUDA: fptest_kat.cu, frtest_kat.cu, g1test_kat.cu, "
                  "fr_fft_testvector.cu, fr_roots.cu",
        "fp": field_kats(os.path.join(REF, "fptest_kat.cu"), "fp"),
        "fr": field_kats(os.path.join(REF, "frtest_kat.cu"), "fr"),
        "g1": g1_kats(os.path.join(REF, "g1test_kat.cu")),
        "fr_fft": fft_vector(os.path.join(REF, "fr_fft_testvector.cu")),
        "fr_roots": roots(os.path.join(REF, "fr_roots.cu")),
    }
    with open(OUT, "w") as f:
        json.dump(data, f, indent=0)
    print("wrote", OUT, {k: (len(v) if isinstance(v, (list, dict)) else v) for k, v in data.items()})


if __name__ == "__main__":
    main()
