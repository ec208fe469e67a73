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


@pytest.mark.parametrize("k", [1, 4, 6])
def test_g_to_lagrange_matches_dft(ctx, k):
    """g_to_lagrange (utils/arithmetic.rs:34-54) against the inverse DFT by
    definition: out[i] = sum_j (n^-1 w^-ij) g[j], one oracle MSM per row."""
    n = 1 << k
    pts = O.gen_bases(120 + k, n)
    dom = mzk.EvaluationDomain(ctx, 5, k)
    d_in, d_out = ctx.alloc(n * 96), ctx.alloc(n * 96)
    d_in.upload(pts)
    dom.g1_to_lagrange_device(d_in, d_out)
    got = d_out.download((n, 12))
    od = O.Domain(5, k)
    w_inv, n_inv = od.get(1), od.get(5)
    for i in range(n):
        wi = O.fr_pow(w_inv, i)
        c = [n_inv]
        for _ in range(n - 1):
            c.append(O.fr_op("mul", c[-1], wi))
        assert np.array_equal(got[i], O.msm_naive(np.stack(c), pts)), i


def test_g_to_lagrange_of_setup_is_setup_lagrange(ctx):
    """Two algorithms, one answer: the inverse FFT of [s^i]G equals the
    Lagrange bases computed from s directly."""
    k = 10
    n = 1 << k
    s = O.rand_fr(130, 1)[0]
    dom, bufs, setup_pts = setup(ctx, k, s)
    out = ctx.alloc(n * 96)
    dom.g1_to_lagrange_device(bufs[0], out)
    assert np.array_equal(out.download((n, 12)), setup_pts[1])


def test_downsize(ctx):
    """ParamsKZG::downsize (params.rs:96-107): the k = 7 bases rebuilt from
    the k = 10 monomial bases equal the k = 7 setup with the same secret."""
    s = O.rand_fr(131, 1)[0]
    _, big, _ = setup(ctx, 10, s)
    small = mzk.EvaluationDomain(ctx, 5, 7)
    n = 1 << 7
    outs = [ctx.alloc(n * 96) for _ in range(3)]
    small.srs_downsize_device(big[0], *outs)
    want = O.srs_setup(s, 7)
    for o, w in zip(outs, want[1:]):
        assert np.array_equal(o.download((n, 12)), w)
