"""KZG test setup on the B200 (ParamsKZG::unsafe_setup, params.rs:160-209,
G1 part) against the oracle, bit-exact, and the relations that tie the SRS to
the MSM and the NTT: one polynomial committed in coefficient form against g,
in Lagrange form against g_lagrange, in delta and double-delta form against
the suffix-sum bases, and [p(s)]G are all the same point."""
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


def setup(ctx, k, s):
    n = 1 << k
    dom = mzk.EvaluationDomain(ctx, 5, k)
    bufs = [ctx.alloc(n * 96) for _ in range(4)]
    dom.srs_setup_device(s, *bufs)
    return dom, bufs, [b.download((n, 12)) for b in bufs]


@pytest.mark.parametrize("k", [1, 4, 8, 10])
def test_srs_matches_oracle(ctx, k):
    s = O.rand_fr(70 + k, 1)[0]
    _, _, got = setup(ctx, k, s)
    want = O.srs_setup(s, k)
    for name, a, b in zip(["g", "g_lagrange", "g_lagrange_delta", "g_lagrange_double_delta"], got, want):
        assert np.array_equal(a, b), name


def test_suffix_sum_with_identity_and_repeats(ctx):
    n = 1000
    pts = O.gen_bases(81, n)
    pts[5] = 0                 # identity
    pts[700] = pts[701]        # equal neighbours: a doubling inside the scan
    pts[999] = pts[998]
    d_in, d_out = ctx.alloc(n * 96), ctx.alloc(n * 96)
    d_in.upload(pts)
    ctx.g1_suffix_sum_device(d_in, n, d_out)
    assert np.array_equal(d_out.download((n, 12)), O.g1_suffix_sum(pts))


def delta(a, order):
    out = a.copy()
    for _ in range(order):
        prev = out.copy()
        for i in range(1, a.shape[0]):
            out[i] = O.fr_op("sub", prev[i], prev[i - 1])
    return out


def test_commitments_agree_across_bases(ctx):
    k = 12
    n = 1 << k
    s = O.rand_fr(90, 1)[0]
    dom, bufs, _ = setup(ctx, k, s)
    coeff = O.rand_fr(91, n)
    lag = dom.coeff_to_lagrange(coeff)
    commits = []
    for scal, base in [(coeff, bufs[0]), (lag, bufs[1]), (delta(lag, 1), bufs[2]), (delta(lag, 2), bufs[3])]:
        d = ctx.alloc(n * 32)
        d.upload(scal)
        commits.append(mzk.affine(ctx.msm_device(d, base, n)))
    trapdoor = O.g1_mul(O.g1_generator(), O.eval_polynomial(coeff, s))
    for c in commits:
        assert np.array_equal(c, trapdoor)
