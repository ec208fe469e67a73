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


def program_lookup(graphs_outs, helpers, agg, mult):
    zero, one = np.zeros(4, np.uint64), O.fr_const(0)
    from _gates import with_constants
    gs = [with_constants(g, zero, one) for g, _ in graphs_outs]
    return gs, {"programs": [as_flat(g) for g in gs], "outputs": [o for _, o in graphs_outs], "helpers": helpers,
                "aggregator": agg, "multiplicities": mult}


@pytest.mark.parametrize("k", [4, 8])
def test_lookup_program_equals_builtin_lookup(ctx, k):
    """The built-in single-input lookup and the same lookup as a helper
    program give the same quotient (with the division), equal to the C oracle."""
    from _gates import single_lookup_graph
    E = 1 << (k + 2)
    cols = make_columns(80 + k, E, 5, 2, lookup_selector=6)
    got_builtin, expect = run_both(ctx, k, cols, True)
    prog = dict(cols)
    lk = prog.pop("lookup")
    _, lp = program_lookup([single_lookup_graph(lk["input"], lk["table"], lk["selector"])], [lk["h"]], lk["z"],
                           lk["m"])
    prog["lookup_programs"] = [lp]
    assert np.array_equal(got_builtin, expect)
    assert np.array_equal(device_quotient(ctx, k, prog, True), expect)


@pytest.mark.parametrize("k", [3, 6])
def test_lookups_and_trash_of_any_shape_match_oracle(ctx, k):
    """Two lookups (one of three inputs in two helper chunks, one
    single-input) and a trashcan after a gate program and two permutation
    sets, against the oracle: the C oracle's gates + permutations (here
    the same gate as a program) continued by the restated lookup and trash
    terms, then divided by t(X)."""
    from _gates import multi_lookup_graphs, single_lookup_graph, standard_gate_graph, trash_graph, with_constants
    ek = k + 2
    E = 1 << ek
    cols = make_columns(90 + k, E, 5, 2, lookup_selector=None)
    cols["trash_challenge"] = O.rand_fr(95 + k, 1)[0]
    col = lambda i: O.rand_fr(9000 + 10 * k + i, E)
    g_multi, lp0 = program_lookup(multi_lookup_graphs(), [col(0), col(1)], col(2), col(3))
    g_single, lp1 = program_lookup([single_lookup_graph(1, 5, 6)], [col(4)], col(5), col(6))
    tg = with_constants(trash_graph(), np.zeros(4, np.uint64), O.fr_const(0))
    trash = {"program": as_flat(tg), "selector": 2, "trash": col(7)}
    base = run_both(ctx, k, cols, False)[1]                      # C oracle: standard gate + permutations
    want = O.flat_tail_eval(base, cols["fixed"], cols["advice"], [], k, ek, cols["beta"], cols["theta"],
                            cols["trash_challenge"], cols["y"], cols["l0"], cols["l_last"], cols["l_active"],
                            lookups=[dict(lp0, programs=g_multi), dict(lp1, programs=g_single)],
                            trashcans=[dict(trash, program=tg)])
    dev_cols = dict(cols)
    dev_cols["gates"] = as_flat(standard_gate_graph())
    dev_cols["lookup_programs"] = [lp0, lp1]
    dev_cols["trash"] = [trash]
    assert np.array_equal(device_quotient(ctx, k, dev_cols, False), want)
    assert np.array_equal(device_quotient(ctx, k, dev_cols, True), O.Domain(5, k).divide_by_vanishing_poly(want))


def test_bad_lookup_and_trash_programs_are_refused(ctx):
    from _gates import single_lookup_graph
    k, E = 3, 1 << 5
    cols = make_columns(7, E, 3, 1, lookup_selector=6)
    lk = cols["lookup"]
    g, outs = single_lookup_graph(0, 5, 6)
    _, lp = program_lookup([(g, outs)], [lk["h"]], lk["z"], lk["m"])
    both = dict(cols, lookup_programs=[lp])                          # built-in lookup and a program
    with pytest.raises(mzk.MzkError):
        device_quotient(ctx, k, both, False)
    c = dict(cols)
    c.pop("lookup")
    _, lp_bad = program_lookup([(g, (1, 11, 13, 14))], [lk["h"]], lk["z"], lk["m"])   # output past values_len
    with pytest.raises(mzk.MzkError):
        device_quotient(ctx, k, dict(c, lookup_programs=[lp_bad]), False)
    from _gates import trash_graph, with_constants
    tg = as_flat(with_constants(trash_graph(), np.zeros(4, np.uint64), O.fr_const(0)))
    with pytest.raises(mzk.MzkError):                                 # selector column 9 of 7
        device_quotient(ctx, k, dict(c, trash=[{"program": tg, "selector": 9, "trash": lk["h"]}]), False)
