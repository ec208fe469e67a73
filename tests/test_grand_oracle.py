"""The oracle's restatements of the permutation grand products
(permutation/prover.rs:81-255), the logup helper and aggregator
(logup/prover.rs:195-300), ff's BatchInvert and kate_division
(utils/arithmetic.rs:106-125), checked against a second, line-by-line
Python restatement on small domains and against the soundness conditions
the reference itself asserts: l_last (z^2 - z) = 0 (the last permutation
product is one when the copy constraints hold) and a zero logup running
sum at the last active row (logup/prover.rs debug assertion)."""
import numpy as np
import pytest

from oracle import oracle as O

ONE = O.fr_const(0)
ZERO = np.zeros(4, np.uint64)
DELTA = O.fr_const(5)


def mul(a, b):
    return O.fr_op("mul", a, b)


def add(a, b):
    return O.fr_op("add", a, b)


def sub(a, b):
    return O.fr_op("sub", a, b)


def small(v):
    return O.fr_op("from_canonical", O.from_int(int(v), 4))


def py_batch_invert(a):
    out = a.copy()
    for i in range(a.shape[0]):
        if a[i].any():
            out[i] = O.fr_op("inv", a[i])
    return out


def py_permutation_z(values, sigmas, chunk_len, k, omega, beta, gamma, bf, blinds):
    n = 1 << k
    sets = [(values[i:i + chunk_len], sigmas[i:i + chunk_len]) for i in range(0, len(values), chunk_len)]
    zs, uncorrected = [], []
    for s, (vals, sigs) in enumerate(sets):
        mv = [ONE.copy() for _ in range(n)]
        for v, sg in zip(vals, sigs):
            for i in range(n):
                mv[i] = mul(mv[i], add(add(mul(beta, sg[i]), gamma), v[i]))
        mv = list(py_batch_invert(np.array(mv)))
        dw0 = O.fr_pow(DELTA, s * chunk_len)
        for v in vals:
            dw = dw0.copy()
            for i in range(n):
                mv[i] = mul(mv[i], add(add(mul(dw, beta), gamma), v[i]))
                dw = mul(dw, omega)
            dw0 = mul(dw0, DELTA)
        z = [ONE.copy()]
        for r in range(1, n):
            z.append(mul(z[r - 1], mv[r - 1]))
        for b in range(bf):
            z[n - bf + b] = blinds[s][b]
        uncorrected.append(z[n - bf - 1])
        zs.append(z)
    corr = ONE.copy()
    out = []
    for s, z in enumerate(zs):
        out.append(np.array([mul(x, corr) for x in z]))
        corr = mul(corr, uncorrected[s])
    return out


def py_logup(chunks, table, selector, m, beta, bf, blinds):
    n = table.shape[0]
    tden = py_batch_invert(np.array([add(beta, t) for t in table]))
    helpers = []
    for ch in chunks:
        h = [ZERO.copy() for _ in range(n)]
        for col in ch:
            inv = py_batch_invert(np.array([add(beta, v) for v in col]))
            h = [add(h[i], inv[i]) for i in range(n)]
        helpers.append(np.array(h))
    agg, state = [ZERO.copy()], ZERO.copy()
    for i in range(n - bf - 1):
        hs = ZERO.copy()
        for h in helpers:
            hs = add(hs, h[i])
        state = add(state, sub(mul(selector[i], hs), mul(m[i], tden[i])))
        agg.append(state)
    agg += list(blinds)
    return helpers, np.array(agg)


def test_batch_invert_skips_zeros():
    a = O.rand_fr(3, 50)
    a[[0, 7, 49]] = 0
    b = O.batch_invert(a)
    assert np.array_equal(b, py_batch_invert(a))
    for i in range(50):
        if a[i].any():
            assert np.array_equal(mul(a[i], b[i]), ONE)
        else:
            assert not b[i].any()


@pytest.mark.parametrize("n", [2, 3, 17, 64])
def test_kate_division(n):
    a = O.rand_fr(10 + n, n)
    b = O.rand_fr(20 + n, 1)[0]
    q = O.kate_division(a, b)
    # a(X) = (X - b) q(X) + a(b): compare coefficients
    r = O.eval_polynomial(a, b)
    rebuilt = [sub(ZERO, mul(b, q[0])) if n > 1 else ZERO.copy()]
    for i in range(1, n - 1):
        rebuilt.append(sub(q[i - 1], mul(b, q[i])))
    rebuilt.append(q[n - 2])
    rebuilt[0] = add(rebuilt[0], r)
    assert np.array_equal(np.array(rebuilt), a)


def omega_of(k):
    return O.Domain(5, k).get(0)


def test_permutation_z_matches_python_restatement():
    k, bf, chunk = 4, 3, 2
    n = 1 << k
    vals = [O.rand_fr(100 + i, n) for i in range(5)]
    sigs = [O.rand_fr(200 + i, n) for i in range(5)]
    beta, gamma = O.rand_fr(300, 1)[0], O.rand_fr(301, 1)[0]
    blinds = O.rand_fr(302, 3 * bf).reshape(3, bf, 4)
    om = omega_of(k)
    got = O.permutation_z(vals, sigs, chunk, k, om, beta, gamma, bf, blinds)
    want = py_permutation_z(vals, sigs, chunk, k, om, beta, gamma, bf, blinds)
    assert len(got) == 3
    for g, w in zip(got, want):
        assert np.array_equal(g, w)


def test_permutation_product_is_one_when_copies_hold():
    """Copy constraints over random cells of the usable rows: the last set's
    z at row n - blinding_factors - 1 is one (l_last (z^2 - z) = 0), and each
    set starts where the previous one ended."""
    k, bf, chunk, ncols = 6, 5, 2, 5
    n, u = 1 << k, (1 << k) - 5 - 1
    rng = np.random.default_rng(7)
    om = omega_of(k)
    # cell (col, row) -> identity label delta^col * omega^row
    ident = [[mul(O.fr_pow(DELTA, c), O.fr_pow(om, r)) for r in range(n)] for c in range(ncols)]
    vals = [O.rand_fr(400 + c, n) for c in range(ncols)]
    sig = [[ident[c][r].copy() for r in range(n)] for c in range(ncols)]
    cells = [(c, r) for c in range(ncols) for r in range(u)]
    rng.shuffle(cells)
    pos = 0
    while pos + 3 <= len(cells) // 3:   # cycles of length 3 over ~1/3 of the cells
        cyc = cells[pos:pos + 3]
        pos += 3
        v = vals[cyc[0][0]][cyc[0][1]].copy()
        for c, r in cyc:
            vals[c][r] = v
        for i, (c, r) in enumerate(cyc):
            c2, r2 = cyc[(i + 1) % 3]
            sig[c][r] = ident[c2][r2]
    sigmas = [np.array(s) for s in sig]
    beta, gamma = O.rand_fr(500, 1)[0], O.rand_fr(501, 1)[0]
    blinds = O.rand_fr(502, 3 * bf).reshape(3, bf, 4)
    zs = O.permutation_z(vals, sigmas, chunk, k, om, beta, gamma, bf, blinds)
    assert np.array_equal(zs[0][0], ONE)
    for s in range(1, len(zs)):
        assert np.array_equal(zs[s][0], zs[s - 1][u])
    assert np.array_equal(zs[-1][u], ONE)


def test_logup_matches_python_restatement():
    n, bf = 16, 3
    chunks = [[O.rand_fr(600, n), O.rand_fr(601, n)], [O.rand_fr(602, n)]]
    table, sel, m = O.rand_fr(603, n), O.rand_fr(604, n), O.rand_fr(605, n)
    beta = O.rand_fr(606, 1)[0]
    chunks[0][1][5] = sub(ZERO, beta)   # a zero denominator, skipped by the batch inversion
    blinds = O.rand_fr(607, bf)
    hg, ag = O.logup(chunks, table, sel, m, beta, bf, blinds)
    hw, aw = py_logup(chunks, table, sel, m, beta, bf, blinds)
    for a, b in zip(hg, hw):
        assert np.array_equal(a, b)
    assert np.array_equal(ag, aw)


def test_logup_running_sum_is_zero_when_lookup_holds():
    k, bf = 7, 6
    n, u = 1 << k, (1 << k) - 6 - 1
    rng = np.random.default_rng(9)
    tvals = [small(v) for v in range(40)]
    table = np.array([tvals[i % 40] if i < 40 else tvals[0] for i in range(n)])
    sel = np.array([ONE if (i < u and rng.random() < 0.8) else ZERO for i in range(n)])
    picks = rng.integers(0, 40, n)
    f = np.array([tvals[p] for p in picks])
    counts = np.zeros(40, int)
    for i in range(u):
        if sel[i].any():
            counts[picks[i]] += 1
    m = np.array([small(counts[i]) if i < 40 else ZERO for i in range(n)])
    beta = O.rand_fr(700, 1)[0]
    blinds = O.rand_fr(701, bf)
    _, agg = O.logup([[f]], table, sel, m, beta, bf, blinds)
    assert not agg[0].any()
    assert not agg[u].any()
    assert np.array_equal(agg[n - bf:], blinds)


def test_poly_inner_product_matches_python():
    polys = [O.rand_fr(800, 7), O.rand_fr(801, 3), O.rand_fr(802, 5)]
    sc = O.rand_fr(803, 3)
    got = O.poly_inner_product(polys, sc)
    want = []
    for i in range(7):
        acc = ZERO.copy()
        for p, s in zip(polys, sc):
            if i < p.shape[0]:
                acc = add(acc, mul(p[i], s))
        want.append(acc)
    assert np.array_equal(got, np.array(want))
