"""g1p_fft_noalloc -- the G1 FFT entry point that allocates no device memory.

It exists for callers that cannot have a library allocate: their device
memory is owned by their own allocator or pool, or they cannot afford the
device-wide synchronisation that cudaMalloc/cudaFree imply.  Its working tiles
live in a fixed device array inside the library, shared by every call.

This file is collected last on purpose (pytest orders files by name), so a run
that stops at the first failure has already run every other test; it also
passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def subgroup_points(engine, seed, count):
    """count points [k_i] G1 for seeded scalars, computed on the GPU."""
    gen = engine.to_device(np.repeat(O.g1_generator().reshape(1, 18), count, 0))
    scal = engine.to_device(O.seeded_fr(seed, count))
    out = engine.empty((count, 18))
    engine.call("g1p_op_n", engine.G1_OPS["mul"], engine._ptr(out), engine._ptr(gen), engine._ptr(scal), count,
                engine._stream())
    return out


def test_noalloc_fft_matches_allocating_entry_point(engine):
    import torch
    lib = engine.lib()
    st = engine._stream()
    # two calls in a row with different shapes: the second must not see the
    # first call's leftovers in the shared scratch array
    for log_m, count, inverse, seed in ((9, 40, 0, 11), (8, 7, 1, 12), (9, 64, 1, 13)):
        m = 1 << log_m
        pts = subgroup_points(engine, seed, count * m).reshape(count, m, 18)
        got = engine.empty((count, m, 18))
        exp = engine.empty((count, m, 18))
        rc = lib.g1p_fft_noalloc(engine._ptr(got), engine._ptr(pts), log_m, count, inverse, st)
        assert rc == 0
        engine.call("g1p_fft_n", engine._ptr(exp), engine._ptr(pts), log_m, count, inverse, st)
        torch.cuda.synchronize()
        assert torch.equal(got, exp), (log_m, count, inverse)


def test_noalloc_fft_rejects_requests_beyond_its_scratch(engine):
    lib = engine.lib()
    pts = engine.empty((65, 512, 18))
    out = engine.empty((65, 512, 18))
    rc = lib.g1p_fft_noalloc(engine._ptr(out), engine._ptr(pts), 9, 65, 0, engine._stream())
    assert rc == engine.FK20_ETOOBIG
    assert lib.g1p_fft_noalloc(engine._ptr(out), engine._ptr(pts), 10, 1, 0, engine._stream()) == engine.FK20_EINVAL


def test_noalloc_fft_matches_oracle(engine):
    """Independent of the allocating entry point: the oracle's G1 FFT
    (the reference's g1p_fft / g1p_ift, g1p_fft.cu:337-350) on a few small
    transforms, forward and inverse, compared after affine normalisation."""
    import torch
    lib = engine.lib()
    st = engine._stream()
    for log_m, count, inverse, seed in ((4, 3, 0, 21), (5, 2, 1, 22)):
        m = 1 << log_m
        pts = subgroup_points(engine, seed, count * m).reshape(count, m, 18)
        got = engine.empty((count, m, 18))
        assert lib.g1p_fft_noalloc(engine._ptr(got), engine._ptr(pts), log_m, count, inverse, st) == 0
        torch.cuda.synchronize()
        host_in = engine.to_host(pts)
        exp = np.stack([O.g1_fft(host_in[k], inverse=bool(inverse)) for k in range(count)])
        norm = lambda a: O.g1_normalize(np.ascontiguousarray(a).reshape(-1, 18)).reshape(count, m, 18)
        assert np.array_equal(norm(engine.to_host(got)), norm(exp)), (log_m, count, inverse)
