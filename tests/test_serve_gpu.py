"""The proving service (continuous batching over create_proof): every
transcript is the one the same proof gets alone, whatever wave it lands in and
whatever mix of sizes shares that wave, and it is the oracle's and verifies;
the plain mode and the memory budget run one proof per wave; bad requests are
refused."""
import threading

import pytest

from _plonk_setup import Circuit, mzk
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = mzk.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def keys(ctx):
    """Keys for k = 5 and k = 7 whose bases live in ONE SRS buffer, each k's
    g | lagrange | delta | double delta at its own offsets."""
    s = O.rand_fr(777, 1)[0]
    sizes = {7: 1 << 7, 5: 1 << 5}
    total = sum(4 * n for n in sizes.values())
    buf = ctx.alloc(total * 96)
    out, at = {"buf": buf}, 0
    for k, n in sizes.items():
        dom = mzk.EvaluationDomain(ctx, 5, k)
        p = buf.ptr + at * 96
        dom.srs_setup_device(s, p, p + n * 96, p + 2 * n * 96, p + 3 * n * 96)
        dom.close()
        offs = (at, at + n, at + 2 * n, at + 3 * n)
        at += 4 * n
        out[k] = offs
    for k in sizes:
        d = mzk.SrsDesc(buf.ptr, total, *out[k], 0, 0, 0)
        out[k] = Circuit(ctx, k, seed=40 + k, srs=(buf, out[k], d, s))
    return out


def alone(ctx, c, blinds):
    return mzk.create_proofs(ctx, [(c.key, c.advice, blinds)])[0]


def test_mixed_waves_equal_alone_and_oracle(ctx, keys):
    srv = mzk.ProvingServer(ctx, max_batch=8)
    jobs = [(keys[k], keys[k].blinds(100 + i)) for i, k in enumerate([5, 7, 7, 5, 5, 7, 5, 7, 7, 5])]
    results = {}

    def client(part):
        tickets = [(i, srv.submit(c.key, c.advice, bl)) for i, (c, bl) in part]
        for i, t in tickets:
            results[i] = srv.wait(t)

    threads = [threading.Thread(target=client, args=(list(enumerate(jobs))[s::2],)) for s in (0, 1)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    stats = srv.stats()
    srv.close()
    assert stats["proofs"] == len(jobs) and 1 <= stats["waves"] <= len(jobs)
    for i, (c, bl) in enumerate(jobs):
        proof, lat = results[i]
        assert lat > 0
        assert proof == alone(ctx, c, bl), i
    for i in (0, 1):                      # one proof of each size: the oracle's transcript, accepted
        c, bl = jobs[i]
        assert results[i][0] == c.oracle_proof(c.advice, bl)
        assert c.verify(results[i][0])


@pytest.mark.parametrize("mode", ["plain", "budget"])
def test_one_proof_per_wave(ctx, keys, mode):
    srv = (mzk.ProvingServer(ctx, max_batch=1, lanes=1, per_call=True) if mode == "plain"
           else mzk.ProvingServer(ctx, max_batch=16, mem_budget_bytes=1))
    c = keys[7]
    bls = [c.blinds(200 + i) for i in range(4)]
    tickets = [srv.submit(c.key, c.advice, bl) for bl in bls]
    outs = [srv.wait(t)[0] for t in tickets]
    stats = srv.stats()
    srv.close()
    assert stats == {"waves": 4, "proofs": 4, "busy_ms": stats["busy_ms"]}
    for bl, o in zip(bls, outs):
        assert o == alone(ctx, c, bl)


def test_bad_requests_are_refused(ctx, keys):
    srv = mzk.ProvingServer(ctx, max_batch=4)
    c = keys[5]
    with pytest.raises(mzk.MzkError):
        srv.submit(c.key, c.advice, c.blinds(1)[:-2])      # wrong number of blinding values
    with pytest.raises(mzk.MzkError):
        srv.wait(12345)                                    # unknown ticket
    # a failing request (a lookup input outside the table) reports its error and the service goes on
    bad = [a.copy() for a in c.advice]
    bad[0][0] = O.rand_fr(5, 1)[0]
    t_bad = srv.submit(c.key, bad, c.blinds(2))
    with pytest.raises(mzk.MzkError, match="not in the table"):
        srv.wait(t_bad)
    assert srv.wait(srv.submit(c.key, c.advice, c.blinds(3)))[0] == alone(ctx, c, c.blinds(3))
    srv.close()
