"""GPU parity of the FK20 pipeline against the oracle (FK20Py restated):
toeplitz coefficients, their FFT, hext_fft, h and every proof h_fft, bit-exact
(canonical limbs, points affine-normalised), for n = 1024, 2048, 4096; the
reference entry points; setup -> xext_fft on the GPU; full-size properties
(KZG identity, linearity); edge cases (zero and non-canonical polynomials,
ragged row counts) and the ragged batch."""
import ctypes

import numpy as np
import pytest

import oracle as O
from conftest import fk20_setup_data

pytestmark = pytest.mark.gpu


def norm(a):
    s = a.shape
    return O.g1_normalize(np.ascontiguousarray(a).reshape(-1, 18)).reshape(s)


_CTX = {}


def ctx_for(engine, n):
    if n not in _CTX:
        _, _, xext = fk20_setup_data(n)
        c = engine.Context(0)
        c.load_xext_fft(n, engine.to_device(xext))
        _CTX[n] = c
    return _CTX[n]


def oracle_rows(poly, xext):
    return [O.fk20_row(poly[r], xext) for r in range(poly.shape[0])]


@pytest.mark.parametrize("n,rows", [(4096, 2), (2048, 3), (1024, 33)])
def test_pipeline_matches_oracle(engine, n, rows):
    m = 2 * n // 16
    _, _, xext = fk20_setup_data(n)
    ctx = ctx_for(engine, n)
    poly = O.seeded_fr(1000 + n, rows * n).reshape(rows, n, 4)
    dpoly = engine.to_device(poly)
    h_fft = engine.empty((rows, m, 18))
    ctx.poly2h_fft(h_fft, dpoly, rows, n)
    hext = engine.empty((rows, m, 18))
    ctx.poly2hext_fft(hext, dpoly, rows, n)
    got_h = norm(engine.to_host(h_fft))
    got_hext = norm(engine.to_host(hext))
    check = [0, rows - 1] if rows > 2 else range(rows)
    exp = O.fk20_rows(poly[list(check)], xext)
    for k, r in enumerate(check):
        assert np.array_equal(got_h[r], exp[k]), f"row {r}"
    ref = O.fk20_row(poly[check[0]], xext)
    assert np.array_equal(got_hext[check[0]], ref["hext_fft"])


def test_reference_entry_points_n4096(engine):
    n, rows, m = 4096, 2, 512
    tau, setup, xext = fk20_setup_data(n)
    poly = O.seeded_fr(4242, rows * n).reshape(rows, n, 4)
    exp = oracle_rows(poly, xext)
    dpoly, dxext = engine.to_device(poly), engine.to_device(xext)
    st = engine._stream()
    P = engine._ptr
    # fk20_poly2h_fft (fk20_poly2h_fft.cu:47), default stream, tables from xext
    h_fft = engine.empty((rows, m, 18))
    engine.call("fk20_poly2h_fft", P(h_fft), P(dpoly), P(dxext), rows)
    import torch
    torch.cuda.synchronize()
    got = norm(engine.to_host(h_fft))
    for r in range(rows):
        assert np.array_equal(got[r], exp[r]["h_fft"])
    # toeplitz -> tc_fft -> msm -> hext_fft2h_fft chained through reference entry points
    tc = engine.empty((rows, 16, m, 4))
    engine.call("fk20_poly2toeplitz_coefficients_fft", P(tc), P(dpoly), rows, st)
    for r in range(rows):
        assert np.array_equal(engine.to_host(tc)[r], exp[r]["tc_fft"])
    hext = engine.empty((rows, m, 18))
    engine.call("fk20_msm", P(hext), P(tc), P(dxext), rows, st)
    for r in range(rows):
        assert np.array_equal(norm(engine.to_host(hext))[r], exp[r]["hext_fft"])
    h2 = engine.empty((rows, m, 18))
    engine.call("fk20_hext_fft2h_fft", P(h2), P(hext), rows, st)
    for r in range(rows):
        assert np.array_equal(norm(engine.to_host(h2))[r], exp[r]["h_fft"])
    # hext_fft -> h (inverse FFT + upper half infinity)
    h = engine.empty((rows, m, 18))
    engine.call("fk20_hext_fft2h", P(h), P(hext), rows, st)
    for r in range(rows):
        assert np.array_equal(norm(engine.to_host(h))[r], exp[r]["h"])
    # h -> h_fft
    engine.call("fk20_h2h_fft", P(h2), P(h), rows, st)
    for r in range(rows):
        assert np.array_equal(norm(engine.to_host(h2))[r], exp[r]["h_fft"])
    # poly -> hext_fft
    engine.call("fk20_poly2hext_fft", P(hext), P(dpoly), P(dxext), rows, st)
    for r in range(rows):
        assert np.array_equal(norm(engine.to_host(hext))[r], exp[r]["hext_fft"])


@pytest.mark.parametrize("n", [1024, 4096])
def test_setup_to_xext_fft_on_gpu(engine, n):
    tau, setup, xext = fk20_setup_data(n)
    m = 2 * n // 16
    dsetup = engine.to_device(setup)
    out = engine.empty((16, m, 18))
    if n == 4096:
        engine.call("fk20_setup2xext_fft", engine._ptr(out), engine._ptr(dsetup), engine._stream())
        assert np.array_equal(norm(engine.to_host(out)), xext)
    # a context built from the setup gives the same proofs as one built from xext
    c = engine.Context(0)
    c.load_setup(n, dsetup)
    rows = 2
    poly = engine.to_device(O.seeded_fr(9, rows * n).reshape(rows, n, 4))
    a, b = engine.empty((rows, m, 18)), engine.empty((rows, m, 18))
    c.poly2h_fft(a, poly, rows, n)
    ctx_for(engine, n).poly2h_fft(b, poly, rows, n)
    assert np.array_equal(norm(engine.to_host(a)), norm(engine.to_host(b)))
    c.close()


def test_kzg_identity_full_batch(engine):
    """512 rows x 4096: sampled proofs equal [q_j(tau)] G1 (pairing-free KZG
    identity with tau known; kzg_proofs.py:198-205)."""
    n, rows, m = 4096, 512, 512
    tau, _, _ = fk20_setup_data(n)
    poly = O.seeded_fr(31337, rows * n).reshape(rows, n, 4)
    h_fft = engine.empty((rows, m, 18))
    ctx_for(engine, n).poly2h_fft(h_fft, engine.to_device(poly), rows, n)
    got = engine.to_host(h_fft)
    rng = np.random.default_rng(0)
    for r, j in [(0, 0), (511, 511), (255, 256)] + [(int(a), int(b)) for a, b in zip(rng.integers(0, rows, 13),
                                                                                   rng.integers(0, m, 13))]:
        direct = O.kzg_direct(poly[r], tau, 16, j, j + 1)[0]
        assert np.array_equal(O.g1_normalize(got[r, j]), direct), (r, j)


def test_linearity_and_edge_cases(engine):
    n, m = 4096, 512
    rows = 35
    ctx = ctx_for(engine, n)
    a = O.seeded_fr(71, rows * n).reshape(rows, n, 4)
    b = O.seeded_fr(72, rows * n).reshape(rows, n, 4)
    s = O.fr_op("add", a.reshape(-1, 4), b.reshape(-1, 4)).reshape(a.shape)
    a[3] = 0  # zero polynomial row
    s[3] = b[3]
    # non-canonical representatives (x + r < 2^256) must give the same proofs
    a_nc = a.copy()
    for k in range(0, n, 97):
        v = O.limbs_to_int(a_nc[5, k]) + O.R
        if v < (1 << 256):
            a_nc[5, k] = O.int_to_limbs(v, 4)
    outs = []
    for p in (a, b, s, a_nc):
        h = engine.empty((rows, m, 18))
        ctx.poly2h_fft(h, engine.to_device(p), rows, n)
        outs.append(h)
    ha, hb, hs, hnc = outs
    import torch
    st = engine._stream()
    cnt = rows * m
    hab = engine.empty((rows, m, 18))
    engine.call("g1p_op_n", engine.G1_OPS["add"], engine._ptr(hab), engine._ptr(ha), engine._ptr(hb), cnt, st)
    eq = torch.zeros(cnt, dtype=torch.uint8, device="cuda")
    engine.call("g1p_eq_n", ctypes.c_void_p(eq.data_ptr()), engine._ptr(hab), engine._ptr(hs), cnt, st)
    assert int(eq.sum()) == cnt
    engine.call("g1p_eq_n", ctypes.c_void_p(eq.data_ptr()), engine._ptr(ha), engine._ptr(hnc), cnt, st)
    assert int(eq.sum()) == cnt
    zero_row = engine.to_host(ha)[3]
    inf = np.zeros(18, np.uint64)
    inf[6] = 1
    assert all(np.array_equal(p, inf) for p in zero_row)


def test_ragged_batch_matches_per_size(engine):
    sizes = [4096, 1024, 2048, 1024, 4096, 2048, 1024]
    polys, poly_off, out_off = [], [], []
    po = oo = 0
    for j, n in enumerate(sizes):
        polys.append(O.seeded_fr(500 + j, n))
        poly_off.append(po)
        out_off.append(oo)
        po += n
        oo += 2 * n // 16
    for n in (1024, 2048, 4096):
        ctx_for(engine, n)
    c = engine.Context(0)
    for n in (1024, 2048, 4096):
        c.load_xext_fft(n, engine.to_device(fk20_setup_data(n)[2]))
    flat = engine.to_device(np.concatenate(polys))
    out = engine.empty((oo, 18))
    c.batch(out, flat, sizes, poly_off, out_off)
    got = norm(engine.to_host(out))
    for j, n in enumerate(sizes):
        m = 2 * n // 16
        h = engine.empty((1, m, 18))
        ctx_for(engine, n).poly2h_fft(h, engine.to_device(polys[j].reshape(1, n, 4)), 1, n)
        assert np.array_equal(got[out_off[j]:out_off[j] + m], norm(engine.to_host(h))[0]), j
    c.close()


def test_invalid_arguments_rejected(engine):
    ctx = ctx_for(engine, 4096)
    h = engine.empty((1, 512, 18))
    p = engine.to_device(np.zeros((1, 4096, 4), np.uint64))
    with pytest.raises(engine.Fk20Error) as e:
        ctx.poly2h_fft(h, p, 1, 3000)  # unsupported length
    assert e.value.code == engine.FK20_EINVAL
    with pytest.raises(engine.Fk20Error) as e:
        ctx.poly2h_fft(h, p, 0, 4096)  # no rows
    assert e.value.code == engine.FK20_EINVAL
    c = engine.Context(0)
    with pytest.raises(engine.Fk20Error) as e:
        c.poly2h_fft(h, p, 1, 4096)  # no tables loaded
    assert e.value.code == engine.FK20_ENOSETUP
    c.close()


def test_fused_and_staged_fft_agree(engine):
    """The persistent stage-fused G1 FFT launch and the launch-per-stage path
    give the same proofs; the fused launch reports no timeout."""
    n, rows, m = 4096, 70, 512
    ctx = ctx_for(engine, n)
    poly = engine.to_device(O.seeded_fr(123, rows * n).reshape(rows, n, 4))
    a, b = engine.empty((rows, m, 18)), engine.empty((rows, m, 18))
    ctx.set(engine.FK20_OPT_FUSED_FFT, 1)
    ctx.poly2h_fft(a, poly, rows, n)
    assert ctx.status() == 0
    ctx.set(engine.FK20_OPT_FUSED_FFT, 0)
    ctx.poly2h_fft(b, poly, rows, n)
    ctx.set(engine.FK20_OPT_FUSED_FFT, 1)
    assert ctx.status() == 0
    import torch
    assert torch.equal(a, b)


def _eq_count(engine, a, b):
    import torch
    cnt = a.numel() // 18
    eq = torch.zeros(cnt, dtype=torch.uint8, device="cuda")
    engine.call("g1p_eq_n", ctypes.c_void_p(eq.data_ptr()), engine._ptr(a), engine._ptr(b), cnt, engine._stream())
    return int(eq.sum()), cnt


def ragged_instances(count, seed):
    """count instances with lengths drawn uniformly from {1024, 2048, 4096}."""
    rng = np.random.default_rng(seed)
    sizes = [int(x) for x in rng.choice([1024, 2048, 4096], count)]
    poly_off, out_off, po, oo = [], [], 0, 0
    for n in sizes:
        poly_off.append(po)
        out_off.append(oo)
        po += n
        oo += n // 8
    return sizes, poly_off, out_off, po, oo


def test_ragged_1000_instances_one_launch_each(engine):
    """1000 instances of lengths drawn from {1024, 2048, 4096} in one call (one
    MSM launch + one persistent G1 FFT launch over three segments) equal the
    plain per-length path, proof by proof."""
    import torch
    sizes, poly_off, out_off, po, oo = ragged_instances(1000, 2024)
    polys = O.seeded_fr(606, po)
    c = engine.Context(0)
    for n in (1024, 2048, 4096):
        c.load_xext_fft(n, engine.to_device(fk20_setup_data(n)[2]))
    dpolys = engine.to_device(polys)
    out = engine.empty((oo, 18))
    c.profile(True)
    c.batch(out, dpolys, sizes, poly_off, out_off)
    prof = c.profile_read()
    c.profile(False)
    assert prof["msm"][1] == 1 and prof["fft_fused"][1] == 1
    assert c.status() == 0
    # per-length reference: the rows of each length as one contiguous plain call
    exp = engine.empty((oo, 18))
    for n in (1024, 2048, 4096):
        idx = [j for j, s in enumerate(sizes) if s == n]
        rows = torch.stack([dpolys[poly_off[j]:poly_off[j] + n] for j in idx])
        h = engine.empty((len(idx), n // 8, 18))
        c.poly2h_fft(h, rows, len(idx), n)
        for r, j in enumerate(idx):
            exp[out_off[j]:out_off[j] + n // 8] = h[r]
    torch.cuda.synchronize()
    assert torch.equal(out, exp)
    # spot-check against the oracle
    for j in (0, 999):
        n = sizes[j]
        ref = O.fk20_row(polys[poly_off[j]:poly_off[j] + n], fk20_setup_data(n)[2])["h_fft"]
        assert np.array_equal(norm(engine.to_host(out[out_off[j]:out_off[j] + n // 8])), ref)
    c.close()


def test_batch_plan_graph_replay(engine):
    """A ragged batch captured once into a CUDA graph (fk20_plan_*) gives the
    same proofs as the direct call, replay after replay, and refuses to replay
    once its tables were rebuilt."""
    import torch
    sizes, poly_off, out_off, po, oo = ragged_instances(70, 99)
    polys = engine.to_device(O.seeded_fr(707, po))
    c = engine.Context(0, 8)
    for n in (1024, 2048, 4096):
        c.load_xext_fft(n, engine.to_device(fk20_setup_data(n)[2]))
    exp = engine.empty((oo, 18))
    c.batch(exp, polys, sizes, poly_off, out_off)
    out = engine.empty((oo, 18))
    plan = engine.Plan(c, out, polys, sizes, poly_off, out_off)
    for _ in range(3):
        out.zero_()
        plan.launch()
        torch.cuda.synchronize()
        assert torch.equal(out, exp)
    c.load_xext_fft(2048, engine.to_device(fk20_setup_data(2048)[2]))
    with pytest.raises(engine.Fk20Error) as e:
        plan.launch()
    assert e.value.code == engine.FK20_ENOSETUP
    plan.close()
    c.close()


def test_launch_shape_options_agree(engine):
    """MSM block sizes and persistent-grid widths change scheduling only."""
    import torch
    n, rows, m = 2048, 45, 256
    ctx = ctx_for(engine, n)
    poly = engine.to_device(O.seeded_fr(808, rows * n).reshape(rows, n, 4))
    ref = engine.empty((rows, m, 18))
    ctx.poly2h_fft(ref, poly, rows, n)
    for opt, val in ((engine.FK20_OPT_MSM_THREADS, 64), (engine.FK20_OPT_MSM_THREADS, 256),
                     (engine.FK20_OPT_FFT_BLOCKS_PER_SM, 1)):
        old = ctx.get(opt)
        ctx.set(opt, val)
        h = engine.empty((rows, m, 18))
        ctx.poly2h_fft(h, poly, rows, n)
        ctx.set(opt, old)
        torch.cuda.synchronize()
        assert torch.equal(h, ref), (opt, val)
    with pytest.raises(engine.Fk20Error):
        ctx.set(engine.FK20_OPT_MSM_THREADS, 96)


def test_profile_work_accounting(engine):
    """The profiler tags each launch with its algorithmic work -- Fp product or
    square 300 limb products, Fr product 136, G1 addition 12, mixed addition
    11, doubling 8 Fp products, a twiddle its chain's doublings and additions
    plus phi -- recomputed here from the program costs; the executed work of
    the same launches (the kernels' cheaper formulas) is below it."""
    MP, MS_X = 300, 234
    n, rows, window, log_m = 1024, 32, 8, 7
    m = 1 << log_m
    c = engine.Context(0, window)
    c.load_xext_fft(n, engine.to_device(fk20_setup_data(n)[2]))
    poly = engine.to_device(O.seeded_fr(77, rows * n).reshape(rows, n, 4))
    h = engine.empty((rows, m, 18))
    c.profile(True)
    c.poly2h_fft(h, poly, rows, n)
    alg, exe = c.profile_read(), c.profile_read_executed()
    c.profile(False)
    c.close()

    def prog(t):
        d, a = engine.program_cost(t)
        return d * 8 * MP + a * 12 * MP + MP if (d or a) else 0

    def stage(s, kind):
        tot = 0
        for b in range(m // 2):
            if kind == 0:
                j = b & ((m >> (s + 1)) - 1)
                tix = ((m - (j << s)) << (9 - log_m)) & 511
            else:
                j = b & ((1 << s) - 1)
                tix = (j << (log_m - 1 - s)) << (9 - log_m)
            tot += 2 * 12 * MP + prog(tix)
        return tot * rows

    fft = sum(stage(s, 0) + stage(s + 1, 1) for s in range(log_m - 1)) + rows * (m // 2) * 12 * MP
    W = -(-129 // window)  # windows per GLV half
    assert alg["fft_fused"][1] == 1 and alg["fft_fused"][2] == pytest.approx(fft, rel=1e-12)
    assert alg["msm"][2] == pytest.approx(rows * m * (16 * 2 * W * 11 * MP + MP), rel=1e-12)
    assert exe["msm"] == pytest.approx(rows * m * (16 * 2 * W * (8 * MP + 2 * MS_X) + MP), rel=1e-12)
    assert 0 < exe["fft_fused"] < 0.95 * alg["fft_fused"][2]
    assert exe["tc_fft"] == alg["tc_fft"][2] > 0


def test_autotune_keeps_results(engine):
    """The autotuner picks a window within the table budget and launch shapes;
    the tuned context still gives the same proofs."""
    n, rows, m = 1024, 40, 128
    c = engine.Context(0, 9)
    c.load_xext_fft(n, engine.to_device(fk20_setup_data(n)[2]))
    poly = engine.to_device(O.seeded_fr(909, rows * n).reshape(rows, n, 4))
    before = engine.empty((rows, m, 18))
    c.poly2h_fft(before, poly, rows, n)
    res = c.autotune(n, rows=64, max_table_bytes=3 << 30)
    # n = 1024: window 11 takes 2.4 GB, 12 takes 4.4 GB (ceil(129 / w) windows per GLV half)
    assert 8 <= res["window"] <= 11 and res["msm_threads"] in (64, 128, 256)
    assert res["ms"] <= res["ms_default"] * 1.05
    assert c.get(engine.FK20_OPT_MSM_THREADS) == res["msm_threads"]
    after = engine.empty((rows, m, 18))
    c.poly2h_fft(after, poly, rows, n)
    assert _eq_count(engine, before, after) == (rows * m, rows * m)
    assert c.status() == 0
    c.close()


@pytest.mark.parametrize("rows", [1, 31, 33, 577])
def test_row_counts_around_group_boundaries(engine, rows):
    """Partial 32-row groups (idle lanes) at small and large row counts:
    sampled proofs of the first, last and a middle row against the KZG
    identity [q_j(tau)] G1."""
    n, m = 4096, 512
    tau, _, _ = fk20_setup_data(n)
    poly = O.seeded_fr(7000 + rows, rows * n).reshape(rows, n, 4)
    h = engine.empty((rows, m, 18))
    ctx_for(engine, n).poly2h_fft(h, engine.to_device(poly), rows, n)
    got = engine.to_host(h)
    for r, j in [(0, 3), (rows - 1, 509), (rows // 2, 256)]:
        direct = O.kzg_direct(poly[r], tau, 16, j, j + 1)[0]
        assert np.array_equal(O.g1_normalize(got[r, j]), direct), (rows, r, j)


def test_bounded_wait_reports_timeout_and_context_recovers(engine):
    """The persistent FFT's readiness waits are bounded: with a short limit and
    one task that never publishes its completion (a flag nothing sets), the
    tasks that read its outputs give up, the call reports FK20_ETIMEOUT through
    fk20_ctx_status, and the context works normally afterwards."""
    import torch
    n, rows, m = 1024, 40, 128
    c = engine.Context(0, 8)
    c.load_xext_fft(n, engine.to_device(fk20_setup_data(n)[2]))
    poly = engine.to_device(O.seeded_fr(8800, rows * n).reshape(rows, n, 4))
    good = engine.empty((rows, m, 18))
    c.poly2h_fft(good, poly, rows, n)
    assert c.status() == 0
    c.set(engine.FK20_OPT_WAIT_LIMIT, 1 << 12)
    c.set(engine.FK20_OPT_TEST_UNPUBLISHED_TASK, 5)  # a first-stage butterfly of row group 1
    bad = engine.empty((rows, m, 18))
    c.poly2h_fft(bad, poly, rows, n)
    assert c.status() == engine.FK20_ETIMEOUT
    c.set(engine.FK20_OPT_TEST_UNPUBLISHED_TASK, -1)
    c.set(engine.FK20_OPT_WAIT_LIMIT, 0)
    again = engine.empty((rows, m, 18))
    c.poly2h_fft(again, poly, rows, n)
    assert c.status() == 0
    torch.cuda.synchronize()
    assert torch.equal(again, good)
    c.close()
