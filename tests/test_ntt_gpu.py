"""EvaluationDomain NTTs on the B200 against the C oracle, bit-exact.

Every operation of proofs/src/poly/domain.rs:249-380 at small and medium k
(the oracle restates the reference's FFTs), the domain constants of
EvaluationDomain::new, and at the 2^24 size of the NTT sweep a round trip plus
spot evaluations of the polynomial by Horner's rule.
"""
import numpy as np
import pytest

from _loader import load
from oracle import oracle as O

mzk = load()
pytestmark = pytest.mark.gpu

OPS = ["coeff_to_lagrange", "lagrange_to_coeff", "coeff_to_extended", "extended_to_coeff",
       "extended_to_lagrange", "divide_by_vanishing_poly"]


@pytest.fixture(scope="module")
def ctx():
    c = mzk.Context(0)
    yield c
    c.close()


def oracle_op(dom, name, a):
    return getattr(dom, name)(a)


@pytest.mark.parametrize("j", [2, 3, 5])
@pytest.mark.parametrize("k", [1, 2, 3, 4, 5, 8, 11, 12, 13, 16])
def test_domain_ops_match_oracle(ctx, j, k):
    if j == 2 and k == 1:
        pytest.skip("extended domain equals the base domain; covered by the other j")
    g = mzk.EvaluationDomain(ctx, j, k)
    o = O.Domain(j, k)
    assert (g.k, g.extended_k) == (o.k, o.extended_k)
    for which, idx in [(0, 0), (1, 1), (2, 2), (3, 8), (4, 3), (5, 4), (6, 5), (7, 6)]:
        assert np.array_equal(g.constant(which), o.get(idx)), which
    for i in range(1 << (g.extended_k - g.k)):
        assert np.array_equal(g.constant(8, i), o.get(7, i))
    n, en = g.n, g.extended_len
    a = O.rand_fr(1000 * j + k, n)
    e = O.rand_fr(2000 * j + k, en)
    for name, x in [("coeff_to_lagrange", a), ("lagrange_to_coeff", a), ("coeff_to_extended", a),
                    ("extended_to_coeff", e), ("extended_to_lagrange", e), ("divide_by_vanishing_poly", e)]:
        got = getattr(g, name)(x)
        assert np.array_equal(got, oracle_op(o, name, x)), name
    g.close()


def test_inputs_are_not_modified_and_lengths_checked(ctx):
    g = mzk.EvaluationDomain(ctx, 5, 6)
    a = O.rand_fr(5, g.extended_len)
    keep = a.copy()
    g.extended_to_lagrange(a)
    assert np.array_equal(a, keep)
    with pytest.raises(mzk.MzkError):
        g.coeff_to_lagrange(O.rand_fr(1, g.n + 1))


def test_special_vectors(ctx):
    k = 10
    g = mzk.EvaluationDomain(ctx, 5, k)
    n = g.n
    zero = np.zeros((n, 4), np.uint64)
    assert not g.coeff_to_lagrange(zero).any()
    one = np.tile(O.fr_const(0), (n, 1))
    # FFT of the constant polynomial 1 is the all-ones vector
    c = np.zeros((n, 4), np.uint64)
    c[0] = O.fr_const(0)
    assert np.array_equal(g.coeff_to_lagrange(c), one)
    # all-ones evaluations are the constant polynomial 1
    assert np.array_equal(g.lagrange_to_coeff(one), c)
    # values equal to r - 1 everywhere (largest canonical element)
    big = np.tile(O.fr_op("neg", O.fr_const(0)), (n, 1))
    o = O.Domain(5, k)
    assert np.array_equal(g.coeff_to_extended(big), o.coeff_to_extended(big))


@pytest.mark.parametrize("k", [18, 20])
def test_medium_sizes_match_oracle(ctx, k):
    g = mzk.EvaluationDomain(ctx, 5, k)
    o = O.Domain(5, k)
    a = O.rand_fr(77 + k, g.n)
    assert np.array_equal(g.coeff_to_lagrange(a), o.coeff_to_lagrange(a))
    ext = g.coeff_to_extended(a)
    assert np.array_equal(ext, o.coeff_to_extended(a))
    assert np.array_equal(g.extended_to_coeff(ext), o.extended_to_coeff(ext))


def test_ntt_2_24_roundtrip_and_spot_evaluations(ctx):
    """NTT sweep at n = 2^24 (2^26 extended): round trips are the identity and
    sampled outputs equal direct evaluations."""
    k = 24
    g = mzk.EvaluationDomain(ctx, 5, k)
    n, en = g.n, g.extended_len
    da = ctx.gen_rand_fr(0x2424, n)
    a = da.download((n, 4))
    d_lag = ctx.alloc(n * 32)
    g.op_device("coeff_to_lagrange", da, d_lag)
    lag = d_lag.download((n, 4))
    d_back = ctx.alloc(n * 32)
    g.op_device("lagrange_to_coeff", d_lag, d_back)
    assert np.array_equal(d_back.download((n, 4)), a)
    d_ext = ctx.alloc(en * 32)
    g.op_device("coeff_to_extended", da, d_ext)
    ext = d_ext.download((en, 4))
    g.op_device("extended_to_coeff", d_ext, d_ext)
    back = d_ext.download((en, 4))
    assert np.array_equal(back[:n], a) and not back[n:].any()
    # spot checks: lag[i] = a(omega^i), ext[i] = a(zeta * ext_omega^i)
    omega, eomega, zeta = g.constant(0), g.constant(2), g.constant(4)
    for i in [0, 1, 12345, n - 1]:
        assert np.array_equal(lag[i], O.eval_polynomial(a, O.fr_pow(omega, i)))
    for i in [0, 7, en - 3]:
        assert np.array_equal(ext[i], O.eval_polynomial(a, O.fr_op("mul", zeta, O.fr_pow(eomega, i))))


def test_ntt_2_24_all_ops_match_oracle_in_full(ctx):
    """The NTT sweep's largest size compared element by element with the
    oracle: coeff_to_lagrange and lagrange_to_coeff at 2^24, coeff_to_extended
    2^24 -> 2^26 and extended_to_coeff at 2^26."""
    import gc
    k = 24
    g = mzk.EvaluationDomain(ctx, 5, k)
    o = O.Domain(5, k)
    n, en = g.n, g.extended_len
    da = ctx.gen_rand_fr(0x2425, n)
    a = da.download((n, 4))
    out = ctx.alloc(en * 32)
    for name in ("coeff_to_lagrange", "lagrange_to_coeff"):
        g.op_device(name, da, out)
        assert np.array_equal(out.download((n, 4)), getattr(o, name)(a)), name
        gc.collect()
    g.op_device("coeff_to_extended", da, out)
    ext = out.download((en, 4))
    want = o.coeff_to_extended(a)
    assert np.array_equal(ext, want)
    del want
    gc.collect()
    de = ctx.gen_rand_fr(0x2426, en)
    e = de.download((en, 4))
    g.op_device("extended_to_coeff", de, out)
    assert np.array_equal(out.download((en, 4)), o.extended_to_coeff(e))


@pytest.mark.parametrize("k,count", [(10, 70), (14, 5), (18, 3)])
def test_batched_domain_ops_equal_single_calls(ctx, k, count):
    """mzk_domain_op_batch_device: every operation 0-3 on `count` device
    polynomials (70: two launches of up to 64 at k = 10) equals one
    mzk_domain_op_device call each, in place as well, and the batch of
    coefficient-to-Lagrange transforms equals the oracle's FFT."""
    g = mzk.EvaluationDomain(ctx, 5, k)
    n, en = g.n, g.extended_len
    sizes = {"coeff_to_lagrange": (n, n), "lagrange_to_coeff": (n, n), "coeff_to_extended": (n, en),
             "extended_to_coeff": (en, en)}
    for name, (li, lo) in sizes.items():
        ins = [ctx.gen_rand_fr(0x5000 + 97 * i + li, li) for i in range(count)]
        outs = [ctx.alloc(lo * 32) for _ in range(count)]
        g.op_batch_device(name, ins, outs)
        for i in (0, count // 2, count - 1):
            want = ctx.alloc(lo * 32)
            g.op_device(name, ins[i], want)
            assert np.array_equal(outs[i].download((lo, 4)), want.download((lo, 4))), (name, i)
        if li == lo:  # in place
            g.op_batch_device(name, ins, ins)
            assert all(np.array_equal(ins[i].download((li, 4)), outs[i].download((lo, 4))) for i in (0, count - 1))
    if k == 10:
        a = ctx.gen_rand_fr(77, n)
        out = ctx.alloc(n * 32)
        g.op_batch_device("coeff_to_lagrange", [a], [out])
        assert np.array_equal(out.download((n, 4)), O.Domain(5, k).coeff_to_lagrange(a.download((n, 4))))
    with pytest.raises(mzk.MzkError):
        g.op_batch_device("extended_to_lagrange", [a if k == 10 else ctx.alloc(en * 32)], [ctx.alloc(n * 32)])
    g.close()
