"""Custom gates of any circuit on the B200 (a flattened gate program as the
reference's FlatGraphEvaluator, proofs/src/plonk/evaluation.rs:148-213,
530-651), bit-exact: the program alone against the oracle's restatement,
with and without the division by the vanishing polynomial; the standard gate
written as a program against the fused kernel's built-in gate and the C
oracle, with permutation sets and a lookup; malformed programs refused."""
import ctypes

import numpy as np
import pytest

from _gates import FIXED, MUL, OPS, READS, sample_graph, standard_gate_graph
from _loader import load
from oracle import oracle as O
from test_quotient_gpu import make_columns, run_both

mzk = load()
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = mzk.Context(0)
    yield c
    c.close()


def as_flat(graph):
    return mzk.build_flat_graph(graph["constants"], graph["rotations"], graph["reads"], graph["ops"],
                                graph["values_len"], graph["beta_idx"], graph["theta_idx"],
                                graph["trash_challenge_idx"], graph["y_idx"], graph["previous_value_idx"],
                                graph["result_idx"])


def device_quotient(ctx, k, cols, divide):
    g = mzk.EvaluationDomain(ctx, 5, k)
    bufs = []

    def dev(a):
        b = ctx.alloc(a.nbytes)
        b.upload(a)
        bufs.append(b)
        return b.ptr

    desc = mzk.build_quotient_desc(cols, k, g.extended_k, dev)
    out = ctx.alloc(g.extended_len * 32)
    g.quotient_eval_device(desc, out, divide)
    return out.download((g.extended_len, 4))


def gate_columns(seed, E):
    col = lambda i: O.rand_fr(seed * 100 + i, E)
    return {"advice": [col(i) for i in range(3)], "fixed": [col(10 + i) for i in range(3)], "instance": [col(20)],
            "l0": col(30), "l_last": col(31), "l_active": col(32), "y": O.rand_fr(seed, 1)[0],
            "beta": O.rand_fr(seed + 1, 1)[0], "gamma": O.rand_fr(seed + 2, 1)[0],
            "theta": O.rand_fr(seed + 3, 1)[0], "trash_challenge": O.rand_fr(seed + 4, 1)[0]}


@pytest.mark.parametrize("k", [3, 6, 9])
def test_program_matches_oracle(ctx, k):
    ek = k + 2
    E = 1 << ek
    cols = gate_columns(k, E)
    c0 = O.rand_fr(50 + k, 1)[0]
    graph = sample_graph(c0)
    cols["gates"] = as_flat(graph)
    want = O.flat_gates_eval(graph, cols["fixed"], cols["advice"], cols["instance"], k, ek, cols["beta"],
                             cols["theta"], cols["trash_challenge"], cols["y"])
    assert np.array_equal(device_quotient(ctx, k, cols, False), want)
    assert np.array_equal(device_quotient(ctx, k, cols, True), O.Domain(5, k).divide_by_vanishing_poly(want))


@pytest.mark.parametrize("k", [4, 8])
def test_standard_gate_program_equals_builtin_gate(ctx, k):
    E = 1 << (k + 2)
    cols = make_columns(70 + k, E, 5, 2, lookup_selector=6)
    got_builtin, expect = run_both(ctx, k, cols, True)
    prog = dict(cols)
    prog["gates"] = as_flat(standard_gate_graph())
    got_prog, _ = run_both(ctx, k, prog, True)
    assert np.array_equal(got_builtin, expect)
    assert np.array_equal(got_prog, expect)


def bad(graph, **change):
    g = dict(graph)
    g.update(change)
    return g


def test_malformed_programs_are_refused(ctx):
    k = 3
    cols = gate_columns(1, 1 << 5)
    base = sample_graph(O.rand_fr(1, 1)[0])
    cases = [
        bad(base, ops=OPS[:-1] + [(MUL, 40, 1, 2, 0)]),             # dst past values_len
        bad(base, ops=OPS[:-1] + [(9, 31, 1, 2, 0)]),               # no such op kind
        bad(base, reads=READS[:-1] + [(FIXED, 7, 0, 15)]),          # fixed column 7 of 3
        bad(base, reads=READS[:-1] + [(FIXED, 0, 5, 15)]),          # rotation index 5 of 3
        bad(base, result_idx=32),                                   # result past values_len
        bad(base, values_len=300),                                  # more than 256 values
    ]
    for g in cases:
        c = dict(cols)
        c["gates"] = as_flat(g)
        with pytest.raises(mzk.MzkError):
            device_quotient(ctx, k, c, False)
    c = dict(cols)
    c["instance"] = []                                              # the program reads instance column 0
    c["gates"] = as_flat(base)
    with pytest.raises(mzk.MzkError):
        device_quotient(ctx, k, c, False)
