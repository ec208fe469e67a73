"""The proving service (continuous batching over the proof core): every
result is the one the same proof gets alone, whatever wave it lands in and
whatever mix of sizes shares that wave; the plain mode and the memory budget
run one proof per wave; bad requests are refused."""
import threading

import numpy as np
import pytest

from _proof_setup import Setup, mzk
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = mzk.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def keys(ctx):
    """Keys for k = 5 and k = 7 whose bases live in ONE SRS buffer:
    [g (2^7) | lagrange_7 | delta_7 | double_delta_7 | lagrange_5 | delta_5 | double_delta_5]."""
    n7, n5 = 1 << 7, 1 << 5
    srs = O.gen_bases(77, 4 * n7 + 3 * n5)
    buf = ctx.alloc(srs.nbytes)
    buf.upload(srs)
    k7 = Setup(ctx, 7, seed=11, shared=(srs, buf.ptr, (0, n7, 2 * n7, 3 * n7)))
    k5 = Setup(ctx, 5, seed=12, shared=(srs, buf.ptr, (0, 4 * n7, 4 * n7 + n5, 4 * n7 + 2 * n5)))
    return {5: k5, 7: k7, "buf": buf}


def alone(setup, job):
    return setup.g.prove_core_device(setup.pk, [job])[0]


def test_mixed_waves_equal_alone_and_oracle(ctx, keys):
    srv = mzk.ProvingServer(ctx, max_batch=8)
    for k in (5, 7):
        srv.add_key(keys[k].g, keys[k].pk)
    jobs = [(k, keys[k].job(100 + i)) for i, k in enumerate([5, 7, 7, 5, 5, 7, 5, 7, 7, 5])]
    results = {}

    def client(part):
        tickets = [(i, srv.submit(k, jb[0])) for i, (k, jb) in part]
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
    for i, (k, (job, w, ch, blinds)) in enumerate(jobs):
        out, lat = results[i]
        assert lat > 0
        assert np.array_equal(out, alone(keys[k], job)), i
    # one proof of each size against the oracle's step-by-step commitments
    for i in (0, 1):
        k, (job, w, ch, blinds) = jobs[i]
        expect = keys[k].oracle(w, ch, blinds)
        for ci in range(len(mzk.PROOF_CORE_COMMITMENTS)):
            assert np.array_equal(mzk.affine(results[i][0][ci]), expect[ci]), (k, ci)


@pytest.mark.parametrize("mode", ["plain", "budget"])
def test_one_proof_per_wave(ctx, keys, mode):
    srv = (mzk.ProvingServer(ctx, max_batch=1, lanes=1, per_call=True) if mode == "plain"
           else mzk.ProvingServer(ctx, max_batch=16, mem_budget_bytes=1))
    srv.add_key(keys[7].g, keys[7].pk)
    jobs = [keys[7].job(200 + i)[0] for i in range(4)]
    tickets = [srv.submit(7, j) for j in jobs]
    outs = [srv.wait(t)[0] for t in tickets]
    stats = srv.stats()
    srv.close()
    assert stats == {"waves": 4, "proofs": 4, "busy_ms": stats["busy_ms"]}
    for j, o in zip(jobs, outs):
        assert np.array_equal(o, alone(keys[7], j))


def test_bad_requests_are_refused(ctx, keys):
    srv = mzk.ProvingServer(ctx, max_batch=4)
    srv.add_key(keys[5].g, keys[5].pk)
    with pytest.raises(mzk.MzkError):
        srv.submit(9, keys[5].job(300)[0])  # no key for k = 9
    with pytest.raises(mzk.MzkError):
        srv.wait(12345)  # unknown ticket
    with pytest.raises(mzk.MzkError):
        srv.add_key(keys[7].g, keys[5].pk)  # key and domain sizes differ
    srv.close()
