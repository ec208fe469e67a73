"""The oracle's quotient restatement against an independent pure-Python
evaluation of the same formula (proofs/src/plonk/evaluation.rs:818-1114) with
Python integers, on tiny domains.  CPU only."""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O

R = 0x73EDA753299D7D483339D80809A1D80553BDA402FFFE5BFEFFFFFFFF00000001
MONT = pow(2, 256, R)
MINV = pow(MONT, -1, R)


def val(x):
    return O.to_int(x) * MINV % R


def mont(v):
    return O.from_int(v % R * MONT % R, 4)


def column(seed, E):
    return O.rand_fr(seed, E)


def python_numerator(cols, k, ek, y, beta, gamma, zeta, ext_omega, divide, tinv):
    E = 1 << ek
    log_scale = ek - k
    delta = val(O.fr_const(5))
    out = []
    rot = lambda idx, r: (idx + (r << log_scale)) % E
    A = [[val(c[i]) for i in range(E)] for c in cols["advice"]]
    F = [[val(c[i]) for i in range(E)] for c in cols["fixed"]]
    S = [[val(c[i]) for i in range(E)] for c in cols["perm_sigma"]]
    Z = [[val(c[i]) for i in range(E)] for c in cols["perm_z"]]
    l0 = [val(cols["l0"][i]) for i in range(E)]
    ll = [val(cols["l_last"][i]) for i in range(E)]
    la = [val(cols["l_active"][i]) for i in range(E)]
    lk = cols.get("lookup")
    if lk:
        H = [val(lk["h"][i]) for i in range(E)]
        LZ = [val(lk["z"][i]) for i in range(E)]
        LM = [val(lk["m"][i]) for i in range(E)]
    bf = cols["blinding_factors"]
    for idx in range(E):
        a, b, c = (A[j][idx] for j in cols["gate_advice"])
        ql, qr, qm, qo, qc = (F[j][idx] for j in cols["gate_fixed"])
        v = (ql * a + qr * b + qm * a * b + qo * c + qc) % R
        if Z:
            v = (v * y + (1 - Z[0][idx]) * l0[idx]) % R
            zl = Z[-1][idx]
            v = (v * y + (zl * zl - zl) * ll[idx]) % R
            for s in range(1, len(Z)):
                v = (v * y + (Z[s][idx] - Z[s - 1][rot(idx, -(bf + 1))]) * l0[idx]) % R
            cur = beta * zeta * pow(ext_omega, idx, R) % R
            pc = cols["perm_cols"]
            for s in range(len(Z)):
                left, right = Z[s][rot(idx, 1)], Z[s][idx]
                for j in range(s * 3, min(s * 3 + 3, len(pc))):
                    kind, ci = pc[j]
                    x = (A if kind == 0 else F)[ci][idx]
                    left = left * (x + beta * S[j][idx] + gamma) % R
                    right = right * (x + cur + gamma) % R
                    cur = cur * delta % R
                v = (v * y + (left - right) * la[idx]) % R
        if lk:
            v = (v * y + LZ[idx] * (l0[idx] + ll[idx])) % R
            f = A[lk["input"]][idx] + beta
            v = (v * y + H[idx] * f - 1) % R
            t = F[lk["table"]][idx] + beta
            sel = 1 if lk["selector"] < 0 else F[lk["selector"]][idx]
            v = (v * y + la[idx] * ((LZ[rot(idx, 1)] - LZ[idx] - sel * H[idx]) * t + LM[idx])) % R
        if divide:
            v = v * tinv[idx & (len(tinv) - 1)] % R
        out.append(v)
    return out


@pytest.mark.parametrize("n_perm,n_sets,sel", [(0, 0, None), (3, 1, -1), (5, 2, 6), (7, 3, 6)])
def test_oracle_quotient_matches_python(n_perm, n_sets, sel):
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parent))
    from test_quotient_gpu import make_columns

    k, j = 2, 5
    d = O.Domain(j, k)
    ek = d.extended_k
    E = 1 << ek
    cols = make_columns(5 + n_sets, E, n_perm, n_sets, sel)
    cols["extended_omega"], cols["g_coset"] = d.get(2), d.get(3)
    keep = []

    def ptrs(items):
        arr = (ctypes.c_void_p * max(1, len(items)))(*[a.ctypes.data for a in items])
        keep.append(arr)
        return ctypes.cast(arr, ctypes.POINTER(ctypes.c_void_p))

    def u32s(items):
        arr = (ctypes.c_uint32 * max(1, len(items)))(*items)
        keep.append(arr)
        return ctypes.cast(arr, ctypes.POINTER(ctypes.c_uint32))

    q = O.QuotientDesc()
    q.k, q.extended_k = k, ek
    q.advice, q.n_advice = ptrs(cols["advice"]), 3
    q.fixed, q.n_fixed = ptrs(cols["fixed"]), 7
    q.gate_fixed[:] = cols["gate_fixed"]
    q.gate_advice[:] = cols["gate_advice"]
    q.n_perm_cols = n_perm
    q.perm_col_kind = u32s([a for a, _ in cols["perm_cols"]])
    q.perm_col_index = u32s([b for _, b in cols["perm_cols"]])
    q.perm_sigma = ptrs(cols["perm_sigma"])
    q.n_perm_sets = n_sets
    q.perm_z = ptrs(cols["perm_z"])
    q.chunk_len, q.blinding_factors = 3, 7
    if sel is not None:
        lk = cols["lookup"]
        q.has_lookup = 1
        q.lookup_input_advice, q.lookup_table_fixed, q.lookup_selector_fixed = 0, 5, sel
        q.lookup_h, q.lookup_z, q.lookup_m = lk["h"].ctypes.data, lk["z"].ctypes.data, lk["m"].ctypes.data
    q.l0, q.l_last, q.l_active = cols["l0"].ctypes.data, cols["l_last"].ctypes.data, cols["l_active"].ctypes.data
    for name in ("y", "beta", "gamma", "theta", "extended_omega", "g_coset"):
        getattr(q, name)[:] = [int(v) for v in cols[name]]
    tinv = [val(d.get(7, i)) for i in range(1 << (ek - k))]
    for divide in (False, True):
        got = d.quotient_eval(q, divide)
        want = python_numerator(cols, k, ek, val(cols["y"]), val(cols["beta"]), val(cols["gamma"]),
                                val(d.get(3)), val(d.get(2)), divide, tinv)
        assert [val(x) for x in got] == want


def test_flat_gates_restatement_matches_direct_evaluation():
    """The oracle's restatement of FlatGraphEvaluator::evaluate_chunk on the
    sample program equals the three gates evaluated directly with Python
    integers (rotations in the extended domain scaled by 2^(ek - k))."""
    from _gates import sample_graph
    k, ek = 3, 5
    E, scale = 1 << ek, ek - k
    fixed = [column(900 + i, E) for i in range(3)]
    advice = [column(910 + i, E) for i in range(3)]
    instance = [column(920, E)]
    c0, y, beta, theta, trash = (O.rand_fr(930 + i, 1)[0] for i in range(5))
    got = O.flat_gates_eval(sample_graph(c0), fixed, advice, instance, k, ek, beta, theta, trash, y)
    F = [[val(c[i]) for i in range(E)] for c in fixed]
    A = [[val(c[i]) for i in range(E)] for c in advice]
    I0 = [val(instance[0][i]) for i in range(E)]
    yv, th, cv = val(y), val(theta), val(c0)
    for idx in range(E):
        nxt, prv = (idx + (1 << scale)) % E, (idx - (1 << scale)) % E
        g1 = F[0][idx] * A[0][idx] * A[1][nxt] + A[2][idx] - cv
        g2 = A[1][idx] ** 2 - 2 * A[0][prv] * F[1][idx]
        g3 = -(A[2][idx] * F[2][idx]) + A[0][nxt] * th + I0[idx]
        assert val(got[idx]) == ((g1 * yv + g2) * yv + g3) % R, idx


def oracle_quotient(cols, k, divide=False):
    """The C oracle's quotient (built-in gate and lookup) for make_columns data."""
    from _loader import load
    mzk = load()
    o = O.Domain(5, k)
    cols = dict(cols)
    cols["extended_omega"], cols["g_coset"] = o.get(2), o.get(3)
    host = mzk.build_quotient_desc(cols, k, o.extended_k, lambda a: a.ctypes.data)
    od = O.QuotientDesc()
    ctypes.memmove(ctypes.byref(od), ctypes.byref(host), ctypes.sizeof(od))
    od._keep = host._keep
    return o.quotient_eval(od, divide)


def test_lookup_program_restatement_matches_builtin_lookup():
    """The oracle's restatement of the lookup terms of any shape
    (evaluation.rs:1034-1090), run on the single-input lookup written as a
    helper program, continues the gate + permutation value of the C oracle to
    exactly the C oracle's value with its built-in lookup."""
    from _gates import single_lookup_graph, with_constants
    from test_quotient_gpu import make_columns
    k = 3
    E = 1 << (k + 2)
    cols = make_columns(61, E, 5, 2, lookup_selector=6)
    full = oracle_quotient(cols, k)
    base_cols = dict(cols)
    lk = base_cols.pop("lookup")
    base = oracle_quotient(base_cols, k)
    graph, outs = single_lookup_graph(lk["input"], lk["table"], lk["selector"])
    graph = with_constants(graph, np.zeros(4, np.uint64), O.fr_const(0))
    tail = O.flat_tail_eval(base, cols["fixed"], cols["advice"], [], k, k + 2, cols["beta"], cols["theta"],
                            np.zeros(4, np.uint64), cols["y"], cols["l0"], cols["l_last"], cols["l_active"],
                            lookups=[{"programs": [graph], "outputs": [outs], "helpers": [lk["h"]],
                                      "aggregator": lk["z"], "multiplicities": lk["m"]}])
    assert np.array_equal(tail, full)
