"""Column scans on the B200 against the oracle, bit-exact: ff BatchInvert,
eval_polynomial, kate_division, the permutation grand products and the
logup helper/aggregator, including zero denominators, chunk edges and the
soundness conditions (last permutation product one, logup running sum zero)."""
import numpy as np
import pytest

from _loader import load
from oracle import oracle as O

mzk = load()
pytestmark = pytest.mark.gpu

ONE = O.fr_const(0)
ZERO = np.zeros(4, np.uint64)
DELTA = O.fr_const(5)


@pytest.fixture(scope="module")
def ctx():
    c = mzk.Context(0)
    yield c
    c.close()


def dev(ctx, a):
    b = ctx.alloc(max(32, a.nbytes))
    b.upload(a)
    return b


@pytest.mark.parametrize("n", [1, 5, 64, 1000, 1 << 16, (1 << 20) + 3])
def test_batch_invert(ctx, n):
    """Up to one wave of blocks: one inversion per block; 2^20 + 3: the block
    totals are batch-inverted first."""
    a = O.rand_fr(n, n)
    a[:: max(1, n // 7)] = 0
    b = dev(ctx, a)
    ctx.batch_invert_device(b, n)
    assert np.array_equal(b.download((n, 4)), O.batch_invert(a))


def test_batch_invert_with_all_zero_blocks(ctx):
    """Blocks whose elements are all zero (their total is the empty product
    one) beside ordinary ones, on the path that inverts the block totals."""
    n = 1 << 20
    a = O.rand_fr(77, n)
    a[:5000] = 0
    a[700000:704096] = 0
    b = dev(ctx, a)
    ctx.batch_invert_device(b, n)
    assert np.array_equal(b.download((n, 4)), O.batch_invert(a))


@pytest.mark.parametrize("n", [1, 2, 63, 64, 65, 4097, 1 << 20])
def test_eval_polynomial(ctx, n):
    a = O.rand_fr(30 + n, n)
    x = O.rand_fr(31 + n, 1)[0]
    assert np.array_equal(ctx.eval_polynomial_device(dev(ctx, a), n, x), O.eval_polynomial(a, x))


def test_eval_polynomial_at_zero_and_one(ctx):
    a = O.rand_fr(40, 300)
    b = dev(ctx, a)
    assert np.array_equal(ctx.eval_polynomial_device(b, 300, ZERO), a[0])
    assert np.array_equal(ctx.eval_polynomial_device(b, 300, ONE), O.eval_polynomial(a, ONE))


@pytest.mark.parametrize("n", [2, 3, 64, 65, 66, 4099, 1 << 18])
def test_kate_division(ctx, n):
    a = O.rand_fr(50 + n, n)
    b = O.rand_fr(51 + n, 1)[0]
    q = ctx.alloc((n - 1) * 32)
    ctx.kate_division_device(dev(ctx, a), n, b, q)
    assert np.array_equal(q.download((n - 1, 4)), O.kate_division(a, b))


def test_kate_division_by_x(ctx):
    a = O.rand_fr(60, 200)
    q = ctx.alloc(199 * 32)
    ctx.kate_division_device(dev(ctx, a), 200, ZERO, q)
    assert np.array_equal(q.download((199, 4)), a[1:])


def perm_case(ctx, k, ncols, chunk, bf, seed):
    n = 1 << k
    dom = mzk.EvaluationDomain(ctx, 5, k)
    vals = [O.rand_fr(seed + c, n) for c in range(ncols)]
    sigs = [O.rand_fr(seed + 100 + c, n) for c in range(ncols)]
    return dom, vals, sigs


@pytest.mark.parametrize("k,ncols,chunk,bf", [(4, 5, 2, 3), (10, 5, 3, 7), (12, 3, 3, 5), (16, 7, 3, 7)])
def test_permutation_z(ctx, k, ncols, chunk, bf):
    n = 1 << k
    dom, vals, sigs = perm_case(ctx, k, ncols, chunk, bf, 1000 + k)
    sets = (ncols + chunk - 1) // chunk
    beta, gamma = O.rand_fr(2000 + k, 1)[0], O.rand_fr(2001 + k, 1)[0]
    vals[0][3] = O.fr_op("sub", ZERO, O.fr_op("add", O.fr_op("mul", beta, sigs[0][3]), gamma))  # zero denominator
    blinds = O.rand_fr(2002 + k, sets * bf).reshape(sets, bf, 4)
    zbufs = [ctx.alloc(n * 32) for _ in range(sets)]
    dom.permutation_z_device([dev(ctx, v) for v in vals], [dev(ctx, s) for s in sigs], chunk, bf, blinds, beta,
                             gamma, zbufs)
    want = O.permutation_z(vals, sigs, chunk, k, O.Domain(5, k).get(0), beta, gamma, bf, blinds)
    for s in range(sets):
        assert np.array_equal(zbufs[s].download((n, 4)), want[s]), s


def test_permutation_product_is_one_when_copies_hold(ctx):
    k, bf, chunk, ncols = 11, 7, 3, 6
    n, u = 1 << k, (1 << k) - bf - 1
    rng = np.random.default_rng(11)
    om = O.Domain(5, k).get(0)
    dpow = [O.fr_pow(DELTA, c) for c in range(ncols)]
    wpow = [ONE]
    for _ in range(n - 1):
        wpow.append(O.fr_op("mul", wpow[-1], om))
    ident = [[O.fr_op("mul", dpow[c], wpow[r]) for r in range(n)] for c in range(ncols)]
    vals = [O.rand_fr(3000 + c, n) for c in range(ncols)]
    sig = [np.array(ident[c]) for c in range(ncols)]
    cells = [(c, r) for c in range(ncols) for r in range(u)]
    order = rng.permutation(len(cells))[: len(cells) // 10 // 4 * 4]
    for g in range(0, len(order), 4):   # cycles of four cells over 10 % of the cells
        cyc = [cells[i] for i in order[g:g + 4]]
        v = vals[cyc[0][0]][cyc[0][1]].copy()
        for c, r in cyc:
            vals[c][r] = v
        for i, (c, r) in enumerate(cyc):
            c2, r2 = cyc[(i + 1) % 4]
            sig[c][r] = ident[c2][r2]
    beta, gamma = O.rand_fr(3100, 1)[0], O.rand_fr(3101, 1)[0]
    sets = 2
    blinds = O.rand_fr(3102, sets * bf).reshape(sets, bf, 4)
    dom = mzk.EvaluationDomain(ctx, 5, k)
    zbufs = [ctx.alloc(n * 32) for _ in range(sets)]
    dom.permutation_z_device([dev(ctx, v) for v in vals], [dev(ctx, s) for s in sig], chunk, bf, blinds, beta, gamma,
                             zbufs)
    z = [b.download((n, 4)) for b in zbufs]
    assert np.array_equal(z[0][0], ONE)
    assert np.array_equal(z[1][0], z[0][u])
    assert np.array_equal(z[1][u], ONE)


@pytest.mark.parametrize("k,bf", [(4, 3), (10, 7), (14, 7)])
def test_logup(ctx, k, bf):
    n = 1 << k
    chunks = [[O.rand_fr(4000 + k, n), O.rand_fr(4001 + k, n)], [O.rand_fr(4002 + k, n)]]
    table, sel, m = O.rand_fr(4003 + k, n), O.rand_fr(4004 + k, n), O.rand_fr(4005 + k, n)
    beta = O.rand_fr(4006 + k, 1)[0]
    chunks[0][1][2] = O.fr_op("sub", ZERO, beta)   # zero denominators stay zero
    table[5] = O.fr_op("sub", ZERO, beta)
    blinds = O.rand_fr(4007 + k, bf)
    dom = mzk.EvaluationDomain(ctx, 5, k)
    hb = [ctx.alloc(n * 32) for _ in chunks]
    ab = ctx.alloc(n * 32)
    dom.logup_device([[dev(ctx, c) for c in ch] for ch in chunks], dev(ctx, table), dev(ctx, sel), dev(ctx, m), bf,
                     blinds, beta, hb, ab)
    hw, aw = O.logup(chunks, table, sel, m, beta, bf, blinds)
    for b, w in zip(hb, hw):
        assert np.array_equal(b.download((n, 4)), w)
    assert np.array_equal(ab.download((n, 4)), aw)


def test_logup_running_sum_is_zero_when_lookup_holds(ctx):
    k, bf = 12, 7
    n, u = 1 << k, (1 << k) - bf - 1
    rng = np.random.default_rng(13)
    tv = np.stack([O.fr_op("from_canonical", O.from_int(v, 4)) for v in range(256)])
    table = tv[np.minimum(np.arange(n), 255)]
    table[256:] = tv[0]
    sel = np.zeros((n, 4), np.uint64)
    on = (np.arange(n) < u) & (rng.random(n) < 0.9)
    sel[on] = ONE
    picks = rng.integers(0, 256, n)
    f = tv[picks]
    counts = np.bincount(picks[on], minlength=256)
    m = np.zeros((n, 4), np.uint64)
    m[:256] = np.stack([O.fr_op("from_canonical", O.from_int(int(c), 4)) for c in counts])
    beta = O.rand_fr(5000, 1)[0]
    blinds = O.rand_fr(5001, bf)
    dom = mzk.EvaluationDomain(ctx, 5, k)
    hb, ab = [ctx.alloc(n * 32)], ctx.alloc(n * 32)
    dom.logup_device([[dev(ctx, f)]], dev(ctx, table), dev(ctx, sel), dev(ctx, m), bf, blinds, beta, hb, ab)
    agg = ab.download((n, 4))
    assert not agg[0].any() and not agg[u].any()
    assert np.array_equal(agg[n - bf:], blinds)


def test_bad_descriptors_raise(ctx):
    dom = mzk.EvaluationDomain(ctx, 5, 4)
    v = ctx.alloc(16 * 32)
    with pytest.raises(mzk.MzkError):
        dom.permutation_z_device([v], [v], 0, 3, np.zeros((1, 3, 4), np.uint64), ZERO, ZERO, [v])  # chunk_len 0
    with pytest.raises(mzk.MzkError):
        dom.permutation_z_device([v], [v], 1, 16, np.zeros((1, 16, 4), np.uint64), ZERO, ZERO, [v])  # bf >= n - 1


@pytest.mark.parametrize("lens", [[5], [64, 17, 64], [1000, 3, 777, 1000, 1], [1 << 16, 1 << 14]])
def test_poly_inner_product(ctx, lens):
    polys = [O.rand_fr(6000 + i + len(lens), n) for i, n in enumerate(lens)]
    scalars = O.rand_fr(6100 + len(lens), len(lens))
    out_len = max(lens)
    out = ctx.alloc(out_len * 32)
    ctx.poly_inner_product_device([dev(ctx, p) for p in polys], lens, scalars, out, out_len)
    assert np.array_equal(out.download((out_len, 4)), O.poly_inner_product(polys, scalars))


def test_multi_open_final_step(ctx):
    """The last step of multi_open (kzg/mod.rs:268-283) through the device
    entry points: final = sum_p x4^p q_p, v = final(x3), pi = (final - v)/(X - x3);
    checked against the oracle's primitives."""
    qs = [O.rand_fr(6200 + i, n) for i, n in enumerate([300, 250, 300])]
    x3, x4 = O.rand_fr(6300, 2)
    pw = [ONE, x4, O.fr_op("mul", x4, x4)]
    final = ctx.alloc(300 * 32)
    ctx.poly_inner_product_device([dev(ctx, q) for q in qs], [300, 250, 300], np.stack(pw), final, 300)
    v = ctx.eval_polynomial_device(final, 300, x3)
    f = final.download((300, 4))
    f[0] = O.fr_op("sub", f[0], v)
    pi = ctx.alloc(299 * 32)
    ctx.kate_division_device(dev(ctx, f), 300, x3, pi)
    ref_final = O.poly_inner_product(qs, np.stack(pw))
    ref_v = O.eval_polynomial(ref_final, x3)
    assert np.array_equal(v, ref_v)
    ref_final[0] = O.fr_op("sub", ref_final[0], ref_v)
    assert np.array_equal(pi.download((299, 4)), O.kate_division(ref_final, x3))
