"""Fused quotient evaluation (evaluate_numerator + divide_by_vanishing_poly)
on the B200 against the oracle's restatement of
proofs/src/plonk/evaluation.rs:818-1114, bit-exact, on seeded random columns.
"""
import ctypes

import numpy as np
import pytest

from _loader import load
from oracle import oracle as O

mzk = load()
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = mzk.Context(0)
    yield c
    c.close()


def make_columns(seed, E, n_perm_cols, n_sets, lookup_selector):
    rnd = iter(range(10_000))
    col = lambda: O.rand_fr(seed * 1000 + next(rnd), E)
    advice = [col() for _ in range(3)]
    fixed = [col() for _ in range(7)]  # q_l q_r q_m q_o q_c t q_lookup
    perm_pool = [(0, 0), (0, 1), (0, 2), (1, 0), (1, 1), (1, 5), (0, 0)]
    cols = {
        "advice": advice, "fixed": fixed, "gate_fixed": [0, 1, 2, 3, 4], "gate_advice": [0, 1, 2],
        "perm_cols": perm_pool[:n_perm_cols], "perm_sigma": [col() for _ in range(n_perm_cols)],
        "perm_z": [col() for _ in range(n_sets)], "chunk_len": 3, "blinding_factors": 7,
        "l0": col(), "l_last": col(), "l_active": col(),
        "y": O.rand_fr(seed, 1)[0], "beta": O.rand_fr(seed + 1, 1)[0], "gamma": O.rand_fr(seed + 2, 1)[0],
        "theta": O.rand_fr(seed + 3, 1)[0],
    }
    if lookup_selector is not None:
        cols["lookup"] = {"input": 0, "table": 5, "selector": lookup_selector, "h": col(), "z": col(), "m": col()}
    return cols


def run_both(ctx, k, cols, divide):
    g = mzk.EvaluationDomain(ctx, 5, k)
    o = O.Domain(5, k)
    E = g.extended_len
    cols = dict(cols)
    cols["extended_omega"], cols["g_coset"] = o.get(2), o.get(3)
    host_desc = mzk.build_quotient_desc(cols, k, g.extended_k, lambda a: a.ctypes.data)
    odesc = O.QuotientDesc()
    ctypes.memmove(ctypes.byref(odesc), ctypes.byref(host_desc), ctypes.sizeof(odesc))
    odesc._keep = host_desc._keep
    expect = o.quotient_eval(odesc, divide)
    bufs = {}

    def dev(a):
        key = id(a)
        if key not in bufs:
            b = ctx.alloc(a.nbytes)
            b.upload(a)
            bufs[key] = (b, a)
        return bufs[key][0].ptr

    desc = mzk.build_quotient_desc(cols, k, g.extended_k, dev)
    out = ctx.alloc(E * 32)
    g.quotient_eval_device(desc, out, divide)
    return out.download((E, 4)), expect


@pytest.mark.parametrize("k", [3, 6, 10])
@pytest.mark.parametrize("n_perm_cols,n_sets", [(3, 1), (5, 2), (7, 3)])
def test_quotient_matches_oracle(ctx, k, n_perm_cols, n_sets):
    E = 1 << (k + 2)
    cols = make_columns(10 * k + n_sets, E, n_perm_cols, n_sets, lookup_selector=6)
    for divide in (False, True):
        got, expect = run_both(ctx, k, cols, divide)
        assert np.array_equal(got, expect), divide


@pytest.mark.parametrize("selector", [None, -1, 6])
def test_quotient_lookup_variants(ctx, selector):
    k = 8
    cols = make_columns(99, 1 << (k + 2), 3, 1, lookup_selector=selector)
    got, expect = run_both(ctx, k, cols, True)
    assert np.array_equal(got, expect)


def test_quotient_gate_only(ctx):
    k = 7
    cols = make_columns(7, 1 << (k + 2), 0, 0, lookup_selector=None)
    got, expect = run_both(ctx, k, cols, True)
    assert np.array_equal(got, expect)


def test_quotient_config3_size(ctx):
    """Extended domain of the k = 18 proof: 2^20 rows."""
    k = 18
    cols = make_columns(18, 1 << 20, 3, 1, lookup_selector=-1)
    got, expect = run_both(ctx, k, cols, True)
    assert np.array_equal(got, expect)


def test_quotient_rejects_mismatched_domain(ctx):
    g = mzk.EvaluationDomain(ctx, 5, 4)
    cols = make_columns(3, 1 << 6, 3, 1, lookup_selector=-1)
    desc = mzk.build_quotient_desc(cols, 5, 7, lambda a: a.ctypes.data)
    with pytest.raises(mzk.MzkError):
        g.quotient_eval_device(desc, ctx.alloc(64 * 32))
