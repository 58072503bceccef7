"""Proofs in the data-availability wire format (48-byte compressed G1, rows in
bit-reversed order; FK20Py/fk20_multi_cuda.py:249-260,
FK20Py/kzg_proofs.py:105-118), against the oracle's restatement of the
format, which is pinned to the published encoding of the generator."""
import numpy as np
import pytest

import oracle as O
from conftest import fk20_setup_data

pytestmark = pytest.mark.gpu


def u8(engine, shape):
    import torch
    return torch.zeros(shape, dtype=torch.uint8, device="cuda")


def test_compress_points(engine):
    import torch
    rng = np.random.default_rng(3)
    g = O.g1_generator().reshape(1, 18)
    ks = [int.from_bytes(rng.bytes(32), "little") % O.R for _ in range(300)]
    pts = O.g1_op("mul", np.repeat(g, len(ks), 0), O.ints_to_array(ks, 4))
    pts = np.concatenate([pts, O.g1_op("neg", pts[:50])])
    inf = np.zeros((1, 18), np.uint64)
    inf[0, 6:12] = [3, 0, 0, 0, 0, 0]  # any (0, y != 0, 0)
    pts = np.concatenate([pts, inf, g])
    # a projective rescaling must not change the encoding
    sc = pts.copy()
    for r in range(0, len(sc), 7):
        if O.limbs_to_int(sc[r, 12:18]) == 0:
            continue
        for c in range(3):
            sc[r, 6 * c:6 * c + 6] = O.int_to_limbs(O.limbs_to_int(sc[r, 6 * c:6 * c + 6]) * 11 % O.P, 6)
    d = engine.to_device(sc)
    out = u8(engine, (len(pts), 48))
    engine.call("fk20_g1p_compress_n", engine._ptr(out), engine._ptr(d), len(pts), engine._stream())
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), O.g1_compress(pts))


@pytest.mark.parametrize("n,rows", [(4096, 2), (1024, 3)])
def test_pipeline_proofs_match_oracle(engine, n, rows):
    import torch
    m = 2 * n // 16
    _, _, xext = fk20_setup_data(n)
    c = engine.Context(0, 8)
    c.load_xext_fft(n, engine.to_device(xext))
    poly = O.seeded_fr(2100 + n, rows * n).reshape(rows, n, 4)
    dpoly = engine.to_device(poly)
    proofs = u8(engine, (rows, m, 48))
    c.poly2proofs(proofs, dpoly, rows, n)
    h = engine.empty((rows, m, 18))
    c.poly2h_fft(h, dpoly, rows, n)
    via_h = u8(engine, (rows, m, 48))
    engine.call("fk20_h_fft2proofs", engine._ptr(via_h), engine._ptr(h), rows, n, engine._stream())
    torch.cuda.synchronize()
    assert torch.equal(proofs, via_h)
    exp = O.da_proofs(np.stack(O.fk20_rows(poly, xext)))
    assert np.array_equal(proofs.cpu().numpy(), exp)
    c.close()


def test_batch_proofs_match_per_instance(engine):
    import torch
    sizes = [4096, 1024, 2048, 1024, 4096]
    po, oo, poly_off, out_off = 0, 0, [], []
    for n in sizes:
        poly_off.append(po)
        out_off.append(oo)
        po += n
        oo += n // 8
    c = engine.Context(0, 8)
    for n in (1024, 2048, 4096):
        c.load_xext_fft(n, engine.to_device(fk20_setup_data(n)[2]))
    polys = engine.to_device(O.seeded_fr(2200, po))
    out = u8(engine, (oo, 48))
    c.batch_proofs(out, polys, sizes, poly_off, out_off)
    for j, n in enumerate(sizes):
        one = u8(engine, (1, n // 8, 48))
        c.poly2proofs(one, polys[poly_off[j]:poly_off[j] + n].reshape(1, n, 4), 1, n)
        torch.cuda.synchronize()
        assert torch.equal(out[out_off[j]:out_off[j] + n // 8], one[0]), j
    c.close()
