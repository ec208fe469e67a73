"""The allocation-free MSM entry point (mzk_msm_g1_noalloc) through the C ABI.

It serves callers that cannot allocate device memory themselves, so it runs
the MSM in a fixed scratch array inside the library.  This file is named to be
collected last: it must pass alone in a fresh process and after every other
test.  Results must be bit-identical to mzk_msm_g1_device on the same device
inputs, on two calls in a row (the second call sees the first call's leftover
scratch contents).
"""
import ctypes

import numpy as np
import pytest

from _loader import load

mzk = load()
pytestmark = pytest.mark.gpu

MAX_N = 1 << 16


@pytest.fixture(scope="module")
def ctx():
    c = mzk.Context(0)
    yield c
    c.close()


def noalloc(ds, db, n, stream=None):
    out = np.zeros(18, np.uint64)
    status = mzk.lib().mzk_msm_g1_noalloc(ds.ptr, db.ptr, n, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), stream)
    mzk._check(status)
    return out


@pytest.mark.parametrize("n", [1000, MAX_N])
def test_noalloc_matches_device_entry_point_twice(ctx, n):
    results = []
    for call, (seed_s, seed_b) in enumerate([(71, 72), (73, 74)]):
        ds = ctx.gen_rand_fr(seed_s + n, n)
        db = ctx.gen_bases(seed_b + n, n)
        expect = ctx.msm_device(ds, db, n)
        got = noalloc(ds, db, n)
        assert np.array_equal(got, expect), f"call {call}"
        results.append(got)
    assert not np.array_equal(results[0], results[1])


def test_noalloc_small_and_empty(ctx):
    ds = ctx.gen_rand_fr(81, 3)
    db = ctx.gen_bases(82, 3)
    assert np.array_equal(noalloc(ds, db, 3), ctx.msm_device(ds, db, 3))
    assert not noalloc(ds, db, 0).any()


def test_noalloc_on_the_context_stream(ctx):
    n = 4096
    ds = ctx.gen_rand_fr(91, n)
    db = ctx.gen_bases(92, n)
    assert np.array_equal(noalloc(ds, db, n, ctx.stream), ctx.msm_device(ds, db, n))


def test_noalloc_rejects_sizes_beyond_its_scratch(ctx):
    ds = ctx.gen_rand_fr(93, 8)
    db = ctx.gen_bases(94, 8)
    out = np.zeros(18, np.uint64)
    status = mzk.lib().mzk_msm_g1_noalloc(ds.ptr, db.ptr, MAX_N + 1, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), None)
    assert status == 1
    assert b"exceeds the fixed scratch limit" in mzk.lib().mzk_last_error()
