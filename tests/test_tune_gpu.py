"""The autotuner on the B200: every NTT pass split computes the same
transform bit for bit (the even split is pinned to the oracle elsewhere;
here every split is also checked against the oracle on a small domain),
autotuned MSM window widths give the same points as the oracle, the table
round-trips through its text file, and malformed input is refused."""
import os

import numpy as np
import pytest

from _loader import load
from oracle import oracle as O

mzk = load()
pytestmark = pytest.mark.gpu

SPLITS = (1, 2, 3)  # even, largest passes first, largest passes last


@pytest.fixture(scope="module")
def ctx():
    c = mzk.Context(0)
    yield c
    c.close()


def set_split(ctx, dom, mode):
    for lg in (dom.k, dom.extended_k):
        ctx.set_tuned(ctx.TUNE_NTT_SPLIT, lg, mode)


@pytest.mark.parametrize("k", [12, 13, 17, 22])
def test_every_split_gives_the_same_transforms(ctx, k):
    dom = mzk.EvaluationDomain(ctx, 5, k)
    a = O.rand_fr(300 + k, dom.n)
    ea = O.rand_fr(400 + k, dom.extended_len)
    set_split(ctx, dom, 0)
    want = [dom.coeff_to_lagrange(a), dom.lagrange_to_coeff(a), dom.coeff_to_extended(a), dom.extended_to_coeff(ea)]
    for mode in SPLITS:
        set_split(ctx, dom, mode)
        got = [dom.coeff_to_lagrange(a), dom.lagrange_to_coeff(a), dom.coeff_to_extended(a), dom.extended_to_coeff(ea)]
        for g, w in zip(got, want):
            assert np.array_equal(g, w), (k, mode)
    set_split(ctx, dom, 0)


@pytest.mark.parametrize("mode", SPLITS)
def test_every_split_matches_the_oracle(ctx, mode):
    k = 13
    dom = mzk.EvaluationDomain(ctx, 5, k)
    od = O.Domain(5, k)
    a = O.rand_fr(77, dom.n)
    set_split(ctx, dom, mode)
    assert np.array_equal(dom.coeff_to_extended(a), od.coeff_to_extended(a))
    assert np.array_equal(dom.lagrange_to_coeff(a), od.lagrange_to_coeff(a))
    set_split(ctx, dom, 0)


def test_autotune_keeps_results(ctx, tmp_path):
    n = 1 << 14
    ds, db = ctx.gen_rand_fr(5, n), ctx.gen_bases(6, n)
    res = ctx.autotune(ds, db, msm_log_n=[12, 14], ntt_log_n=[12, 16], reps=1)
    for L in (12, 14):
        c, ms = res["msm"][L]
        model = mzk.lib().mzk_msm_pick_window(1 << L)
        assert max(5, model - 2) <= c <= model + 2 and ms > 0
    for L in (12, 16):
        assert res["ntt"][L][0] in SPLITS and res["ntt"][L][1] > 0
    # the tuned widths give the oracle's points, single and batched
    s, b = O.rand_fr(5, n), O.gen_bases(6, n)
    s12, b12 = s[:1 << 12], b[:1 << 12]
    assert np.array_equal(mzk.affine(ctx.msm_device(ds, db, 1 << 12)), O.msm_best(s12, b12))
    assert np.array_equal(mzk.affine(ctx.msm_device(ds, db, n)), O.msm_best(s, b))
    out = ctx.msm_batch_device(db, n, [(ds, 0, 1 << 12), (ds, 0, n)])
    assert np.array_equal(mzk.affine(out[0]), O.msm_best(s12, b12))
    assert np.array_equal(mzk.affine(out[1]), O.msm_best(s, b))
    # save, load into a fresh context (and through MZK_TUNE_FILE)
    path = tmp_path / "tune.txt"
    ctx.save_tuning(path)
    text = path.read_text()
    assert f"msm_c 14 {res['msm'][14][0]}" in text and f"ntt_split 16 {res['ntt'][16][0]}" in text
    c2 = mzk.Context(0)
    c2.load_tuning(path)
    assert c2.tuned(c2.TUNE_MSM_WINDOW, 14) == res["msm"][14][0]
    c2.close()
    os.environ["MZK_TUNE_FILE"] = str(path)
    try:
        c3 = mzk.Context(0)
        assert c3.tuned(c3.TUNE_NTT_SPLIT, 16) == res["ntt"][16][0]
        c3.close()
    finally:
        del os.environ["MZK_TUNE_FILE"]
    for kind, L in ((ctx.TUNE_MSM_WINDOW, 12), (ctx.TUNE_MSM_WINDOW, 14), (ctx.TUNE_NTT_SPLIT, 12),
                    (ctx.TUNE_NTT_SPLIT, 16)):
        ctx.set_tuned(kind, L, 0)


def test_bad_tuning_input_is_refused(ctx, tmp_path):
    with pytest.raises(mzk.MzkError):
        ctx.set_tuned(ctx.TUNE_MSM_WINDOW, 14, 30)     # width out of range
    with pytest.raises(mzk.MzkError):
        ctx.set_tuned(ctx.TUNE_NTT_SPLIT, 14, 4)       # no such split
    with pytest.raises(mzk.MzkError):
        ctx.set_tuned(7, 14, 1)                        # no such kind
    with pytest.raises(mzk.MzkError):
        ctx.tuned(ctx.TUNE_MSM_WINDOW, 40)             # no such size slot
    ctx.set_tuned(ctx.TUNE_MSM_WINDOW, 10, 9)
    bad = tmp_path / "bad.txt"
    bad.write_text("msm_c 10 12\nntt_split 11 2 extra\n")
    with pytest.raises(mzk.MzkError):
        ctx.load_tuning(bad)
    assert ctx.tuned(ctx.TUNE_MSM_WINDOW, 10) == 9     # unchanged by the rejected file
    with pytest.raises(mzk.MzkError):
        ctx.load_tuning(tmp_path / "missing.txt")
    os.environ["MZK_TUNE_FILE"] = str(bad)
    try:
        with pytest.raises(mzk.MzkError):
            mzk.Context(0)
    finally:
        del os.environ["MZK_TUNE_FILE"]
    with pytest.raises(mzk.MzkError):
        ctx.autotune(msm_log_n=[12])                  # MSM sizes need device inputs
    ctx.set_tuned(ctx.TUNE_MSM_WINDOW, 10, 0)
