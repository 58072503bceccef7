"""The continuous-batching request server (fk20_server_*): requests of mixed
lengths submitted while others are on the GPU are packed and overlapped, and
every result is bit-identical to proving that polynomial alone."""
import time

import numpy as np
import pytest

import oracle as O
from conftest import fk20_setup_data

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def served_ctx(engine):
    c = engine.Context(0, 8)
    for n in (1024, 2048, 4096):
        c.load_xext_fft(n, engine.to_device(fk20_setup_data(n)[2]))
    yield c
    c.close()


@pytest.mark.parametrize("mode", [{}, {"latency_rows": 4}, {"fft_blocks_per_sm": 1}, {"engine": 1},
                                  {"engine": 1, "cohort_rows": 32, "stages_per_launch": 1, "form_ms": 2},
                                  {"engine": 1, "cohort_rows": 128, "stages_per_launch": 17, "cohorts": 3}],
                         ids=["adaptive", "latency-rows-4", "one-fft-block-per-sm", "cohorts",
                              "cohorts-1-stage-per-launch", "cohorts-whole-fft-per-launch"])
def test_server_results_same_alone_and_in_the_mix(engine, served_ctx, mode):
    """Latency-mode packs (the whole queue, the whole GPU) and throughput-mode
    packs (whole 32-row groups, the SMs split between slots) both occur here:
    bursts of 10 submissions against 16-request packs."""
    rng = np.random.default_rng(5)
    sizes = [int(x) for x in rng.choice([1024, 2048, 4096], 90, p=[0.2, 0.3, 0.5])]
    polys = [O.seeded_fr(4000 + j, n) for j, n in enumerate(sizes)]
    outs = [np.zeros((n // 8, 18), np.uint64) for n in sizes]
    srv = engine.Server(served_ctx, max_rows=16, slots=2, **mode)
    tickets = []
    for j, n in enumerate(sizes):  # arrivals spread over time, so packs overlap with new arrivals
        tickets.append(srv.submit(polys[j], outs[j]))
        if j % 10 == 9:
            time.sleep(0.002)
    deadline = time.time() + 120  # bounded: a stuck server fails the test instead of hanging it
    for t in tickets:
        assert srv.wait(t, max(1, int(1000 * (deadline - time.time())))) == 0
    st = srv.stats()
    assert st["requests"] == len(sizes) and st["proofs"] == sum(n // 8 for n in sizes)
    # engine 0: packs of at most 16 requests; engine 1: at least one cohort per length
    assert st["packs"] >= (3 if mode.get("engine") else len(sizes) // 16)
    assert 0 < st["p50_ms"] <= st["p99_ms"] <= st["max_ms"]
    srv.close()
    # each result equals that polynomial proved alone
    for j, n in enumerate(sizes):
        h = engine.empty((1, n // 8, 18))
        served_ctx.poly2h_fft(h, engine.to_device(polys[j].reshape(1, n, 4)), 1, n)
        assert np.array_equal(engine.to_host(h)[0], outs[j]), j
    # and the proofs are the oracle's
    for j in (0, len(sizes) - 1):
        exp = O.fk20_row(polys[j], fk20_setup_data(sizes[j])[2])["h_fft"]
        assert np.array_equal(O.g1_normalize(outs[j]), exp)


def test_server_rejects_bad_requests(engine, served_ctx):
    srv = engine.Server(served_ctx, max_rows=8, slots=1)
    bad = np.zeros((3000, 4), np.uint64)
    with pytest.raises(engine.Fk20Error) as e:
        srv.submit(bad, np.zeros((375, 18), np.uint64))
    assert e.value.code == engine.FK20_EINVAL
    with pytest.raises(engine.Fk20Error) as e:
        engine.Server(served_ctx, max_rows=8, latency_rows=9)  # latency_rows above max_rows
    assert e.value.code == engine.FK20_EINVAL
    assert srv.wait(12345, 0) == engine.FK20_EINVAL
    p = O.seeded_fr(1, 1024)
    o = np.zeros((128, 18), np.uint64)
    t = srv.submit(p, o)
    assert srv.wait(t, 30000) == 0
    assert srv.wait(t, 0) == engine.FK20_EINVAL  # already collected
    srv.close()


def test_server_without_tables_for_a_length(engine):
    c = engine.Context(0, 8)
    c.load_xext_fft(1024, engine.to_device(fk20_setup_data(1024)[2]))
    srv = engine.Server(c, max_rows=4, slots=1)
    with pytest.raises(engine.Fk20Error) as e:
        srv.submit(O.seeded_fr(2, 4096), np.zeros((512, 18), np.uint64))
    assert e.value.code == engine.FK20_ENOSETUP
    srv.close()
    c.close()


def test_server_close_finishes_pending_requests(engine, served_ctx):
    """Closing the server completes every request already submitted."""
    sizes = [1024, 4096, 2048] * 7
    polys = [O.seeded_fr(4500 + j, n) for j, n in enumerate(sizes)]
    outs = [np.zeros((n // 8, 18), np.uint64) for n in sizes]
    srv = engine.Server(served_ctx, max_rows=8, slots=2)
    for j in range(len(sizes)):
        srv.submit(polys[j], outs[j])
    srv.close()  # returns once the worker has written every result
    for j in (0, 10, len(sizes) - 1):
        n = sizes[j]
        h = engine.empty((1, n // 8, 18))
        served_ctx.poly2h_fft(h, engine.to_device(polys[j].reshape(1, n, 4)), 1, n)
        assert np.array_equal(engine.to_host(h)[0], outs[j]), j


def test_server_memory_budget_limits_packs(engine, served_ctx):
    """Admission by device memory: with a budget of 20 MiB for both slots'
    buffers, the 40 requests submitted at once cannot form one pack (a pack
    of all three lengths needs ~19 MB of scalar and point tiles -- 10.7, 5.4
    and 2.7 MB for the 32-row groups of 4096, 2048 and 1024 coefficients --
    plus ~5 MB of staged inputs and outputs); they are proved in several,
    every one of them exact."""
    rng = np.random.default_rng(8)
    sizes = [int(x) for x in rng.choice([1024, 2048, 4096], 40, p=[0.3, 0.3, 0.4])]
    polys = [O.seeded_fr(6000 + j, n) for j, n in enumerate(sizes)]
    outs = [np.zeros((n // 8, 18), np.uint64) for n in sizes]
    srv = engine.Server(served_ctx, max_rows=64, slots=2, hbm_budget=20 << 20)
    tickets = [srv.submit(polys[j], outs[j]) for j in range(len(sizes))]
    deadline = time.time() + 120
    for t in tickets:
        assert srv.wait(t, max(1, int(1000 * (deadline - time.time())))) == 0
    st = srv.stats()
    srv.close()
    assert st["requests"] == len(sizes) and st["nomem"] == 0
    assert st["packs"] >= 2 and st["mean_pack_rows"] < len(sizes)
    for j, n in enumerate(sizes):
        h = engine.empty((1, n // 8, 18))
        served_ctx.poly2h_fft(h, engine.to_device(polys[j].reshape(1, n, 4)), 1, n)
        assert np.array_equal(engine.to_host(h)[0], outs[j]), j


def test_server_full_queue_refuses_with_eagain(engine, served_ctx):
    """With max_queue requests waiting, submit refuses with FK20_EAGAIN (the
    caller retries later) and counts the refusal; admitted requests are
    proved exactly."""
    srv = engine.Server(served_ctx, max_rows=1, slots=1, max_queue=4)
    polys = [O.seeded_fr(7000 + j, 4096) for j in range(24)]
    outs = [np.zeros((512, 18), np.uint64) for _ in polys]
    admitted, refused = [], 0
    for j in range(len(polys)):
        try:
            admitted.append((j, srv.submit(polys[j], outs[j])))
        except engine.Fk20Error as e:
            assert e.code == engine.FK20_EAGAIN
            refused += 1
    assert refused >= 1 and len(admitted) >= 4
    deadline = time.time() + 120
    for _, t in admitted:
        assert srv.wait(t, max(1, int(1000 * (deadline - time.time())))) == 0
    assert srv.stats()["rejected"] == refused
    srv.close()
    for j, _ in admitted[:3] + admitted[-1:]:
        h = engine.empty((1, 512, 18))
        served_ctx.poly2h_fft(h, engine.to_device(polys[j].reshape(1, 4096, 4)), 1, 4096)
        assert np.array_equal(engine.to_host(h)[0], outs[j]), j
