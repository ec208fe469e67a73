"""Batched MSMs over one shared device SRS against per-item oracle MSMs.

Shapes follow the batched configuration: sizes log-uniform over a range,
one in four sparse (90 % of scalars in {0, 1}), all reading prefixes (or
offset slices) of one resident base array; each result bit-exact.
"""
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


def sparse(s, seed):
    rng = np.random.default_rng(seed)
    u = rng.random(s.shape[0])
    s = s.copy()
    s[u < 0.45] = 0
    s[(u >= 0.45) & (u < 0.9)] = O.fr_const(0)
    return s


def test_batch_matches_oracle(ctx):
    srs_n = 1 << 14
    bases = O.gen_bases(0xB45E, srs_n)
    d_bases = ctx.alloc(bases.nbytes)
    d_bases.upload(bases)
    rng = np.random.default_rng(4)
    items, host = [], []
    keep = []
    for m in range(24):
        n = int(2 ** rng.uniform(4, 14))
        off = int(rng.integers(0, srs_n - n + 1)) if m % 5 == 4 else 0
        s = O.rand_fr(500 + m, n)
        if m % 4 == 3:
            s = sparse(s, m)
        ds = ctx.alloc(s.nbytes)
        ds.upload(s)
        keep.append(ds)
        items.append((ds, off, n))
        host.append((s, bases[off:off + n]))
    items.append((keep[0], 0, 0))  # an empty item gives the identity
    got = ctx.msm_batch_device(d_bases, srs_n, items)
    for m, (s, b) in enumerate(host):
        assert np.array_equal(mzk.affine(got[m]), O.msm_best(s, b)), m
    assert not got[-1].any()


def test_batch_equals_single_calls_and_is_order_independent(ctx):
    srs_n = 1 << 16
    d_bases = ctx.gen_bases(0x5125, srs_n)
    sizes = [1 << 16, 1 << 12, 3000, 1 << 10, 77]
    ds = [ctx.gen_rand_fr(900 + i, n) for i, n in enumerate(sizes)]
    items = [(d, 0, n) for d, n in zip(ds, sizes)]
    got = ctx.msm_batch_device(d_bases, srs_n, items)
    for i, n in enumerate(sizes):
        assert np.array_equal(got[i], ctx.msm_device(ds[i], d_bases, n))
    rev = ctx.msm_batch_device(d_bases, srs_n, items[::-1])
    assert np.array_equal(rev[::-1], got)


def test_batch_rejects_out_of_range_items(ctx):
    d_bases = ctx.gen_bases(1, 64)
    d_s = ctx.gen_rand_fr(2, 64)
    with pytest.raises(mzk.MzkError):
        ctx.msm_batch_device(d_bases, 64, [(d_s, 10, 60)])


def test_config4_batch_at_full_sizes_matches_closed_form(ctx):
    """The batched configuration at its own sizes: 64 MSMs of 2^U(12, 22)
    points over one 2^22-point SRS of bases [r_i]G, one in four sparse (90 %
    of scalars in {0, 1}).  Every item equals [sum_i s_i r_i]G (the scalar
    inner product by the oracle, then one scalar multiplication of G), over
    the plain SRS and over a width-20 window table of it (items of 2^18
    points and more use the table)."""
    srs_n, seed = 1 << 22, 0x5126
    d_bases = ctx.gen_bases(seed, srs_n)
    r = O.rand_fr(seed, srs_n)                       # the bases' discrete logs: the same stream
    rng = np.random.default_rng(0xC4)
    items, want, keep = [], [], []
    g = O.g1_generator()
    for m in range(64):
        n = int(2 ** rng.uniform(12, 22))
        d = ctx.gen_rand_fr(0xB100 + m, n)
        s = d.download((n, 4))
        if m % 4 == 3:
            s = sparse(s, m)
            d.upload(s)
        keep.append(d)
        items.append((d, 0, n))
        want.append(O.g1_mul(g, O.fr_inner_product(s, r[:n])))
    got = ctx.msm_batch_device(d_bases, srs_n, items)
    for m in range(64):
        assert np.array_equal(mzk.affine(got[m]), want[m]), m
    c, rows = 20, mzk.Context.msm_table_rows(20)
    table = ctx.alloc(rows * srs_n * 96)
    ctx.gen_bases(seed, srs_n, out=table)
    del d_bases
    ctx.msm_window_table(table, srs_n, c, rows)
    tabled = ctx.msm_batch_table_device(table, srs_n, c, rows, 1 << 18, items)
    assert np.array_equal(tabled, got)
