"""Fixed-base window tables for a resident SRS on the B200, bit-exact: the
table rows are [2^(c j)] of every base (checked with the oracle's scalar
multiplication), batched MSMs over a table equal the same MSMs without it
(items above and below the size threshold, sparse and zero scalars, an
identity base), and the proof core gives the same commitments with its SRS
as a table, batched and one MSM per call."""
import numpy as np
import pytest

from _loader import load
from _proof_setup import Setup
from oracle import oracle as O

mzk = load()
pytestmark = pytest.mark.gpu
R = 0x73EDA753299D7D483339D80809A1D80553BDA402FFFE5BFEFFFFFFFF00000001


@pytest.fixture(scope="module")
def ctx():
    c = mzk.Context(0)
    yield c
    c.close()


def make_table(ctx, bases, c):
    n, rows = bases.shape[0], mzk.Context.msm_table_rows(c)
    t = ctx.alloc(rows * n * 96)
    t.upload(bases)                                  # row 0
    ctx.msm_window_table(t, n, c, rows)
    return t, rows


def mont_scalar(v):
    return O.fr_op("from_canonical", O.from_int(v % R, 4))


@pytest.mark.parametrize("c", [13, 20])
def test_rows_are_powers_of_two_multiples(ctx, c):
    n = 512
    bases = O.gen_bases(61, n)
    bases[9] = 0                                     # the identity stays the identity
    t, rows = make_table(ctx, bases, c)
    assert rows * c >= 256                           # enough windows for a 255-bit scalar and its carry
    tab = t.download((rows, n, 12))
    assert np.array_equal(tab[0], bases)
    for j in (1, 2, rows - 1):
        for i in (0, 9, 100, n - 1):
            want = O.g1_mul(bases[i], mont_scalar(1 << (c * j))) if bases[i].any() else np.zeros(12, np.uint64)
            assert np.array_equal(tab[j, i], want), (j, i)


@pytest.mark.parametrize("c,min_n", [(16, 1000), (20, 1)])
def test_batch_over_table_equals_plain_batch(ctx, c, min_n):
    n = 1 << 16
    bases = O.gen_bases(62, n)
    bases[3] = 0
    t, rows = make_table(ctx, bases, c)
    plain = ctx.alloc(bases.nbytes)
    plain.upload(bases)
    sizes = [(n, 0), (1 << 14, 100), (3000, 7), (999, 11), (1, 0), (0, 5), (20000, 40000)]
    items = []
    for i, (m, off) in enumerate(sizes):
        s = O.rand_fr(700 + i, max(m, 1))[:m] if m else np.zeros((0, 4), np.uint64)
        if i == 1:
            s[::3] = 0                               # sparse: a third zero, a third one
            s[1::3] = O.fr_const(0)
        if i == 2:
            s[:] = 0                                 # all zero
        d = ctx.alloc(max(32, s.nbytes))
        if m:
            d.upload(s)
        items.append((d, off, m))
    want = ctx.msm_batch_device(plain, n, items)
    got = ctx.msm_batch_table_device(t, n, c, rows, min_n, items)
    assert np.array_equal(got, want)
    assert not got[2].any()                          # all-zero scalars: the identity


def test_prove_core_with_table(ctx):
    st = Setup(ctx, 8, seed=77)
    jobs = [st.job(s)[0] for s in (81, 82)]
    want = st.g.prove_core_device(st.pk, jobs)
    c = 16
    t, rows = make_table(ctx, st.srs, c)
    pk = st.pk
    saved = (pk.srs, pk.srs_table_c, pk.srs_table_rows, pk.srs_table_min_n)
    pk.srs, pk.srs_table_c, pk.srs_table_rows, pk.srs_table_min_n = t.ptr, c, rows, 1
    try:
        assert np.array_equal(st.g.prove_core_device(pk, jobs), want)
        assert np.array_equal(st.g.prove_core_device(pk, jobs, per_call=True), want)
    finally:
        pk.srs, pk.srs_table_c, pk.srs_table_rows, pk.srs_table_min_n = saved


def test_bad_tables_are_refused(ctx):
    bases = O.gen_bases(63, 64)
    t, rows = make_table(ctx, bases, 16)
    d = ctx.alloc(64 * 32)
    d.upload(O.rand_fr(1, 64))
    with pytest.raises(mzk.MzkError):
        ctx.msm_batch_table_device(t, 64, 16, rows - 1, 1, [(d, 0, 64)])   # too few rows for width 16
    with pytest.raises(mzk.MzkError):
        ctx.msm_window_table(t, 64, 16, 3)                                 # fewer rows than the windows
    with pytest.raises(mzk.MzkError):
        ctx.msm_window_table(t, 64, 30, rows)                              # width outside [5, 24]


@pytest.mark.parametrize("c", [12, 16, 18])
def test_served_proofs_over_a_table_equal_the_untabled_proof(ctx, c):
    """create_proof through the proving service with a key whose SRS is a
    window table (the widths prover_table_width gives): every transcript
    equals the same proof with the key over the plain SRS (and the
    oracle's)."""
    from _plonk_setup import PINNED, Circuit
    c8 = Circuit(ctx, 8, seed=91)
    n = c8.n
    blinds = [c8.blinds(s) for s in (92, 93, 94)]
    want = [mzk.create_proofs(ctx, [(c8.key, c8.advice, b)])[0] for b in blinds]
    t, rows = make_table(ctx, c8.srs_buf.download((4 * n, 12)), c)
    desc = mzk.SrsDesc(t.ptr, 4 * n, 0, n, 2 * n, 3 * n, c, rows, 1)
    key = mzk.PlonkKey(ctx, c8.dom, c8.circuit, desc, c8.fixed, c8.mapping, PINNED)
    assert np.array_equal(key.fixed_coms, c8.key.fixed_coms) and np.array_equal(key.repr, c8.key.repr)
    srv = mzk.ProvingServer(ctx, max_batch=4)
    tickets = [srv.submit(key, c8.advice, b) for b in blinds]
    outs = [srv.wait(tk)[0] for tk in tickets]
    srv.close()
    assert outs == want
    assert outs[0] == c8.oracle_proof(c8.advice, blinds[0])
