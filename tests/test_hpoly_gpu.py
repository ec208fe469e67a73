"""compute_h_poly on the device (proofs/src/plonk/prover.rs:701-771) against
the oracle: quotient, division by t(X), extended_to_coeff, limb split with the
same blinds, and one MSM per limb against the monomial SRS; bit-exact."""
import ctypes
import sys
from pathlib import Path

import numpy as np
import pytest

from _loader import load
from oracle import oracle as O

sys.path.insert(0, str(Path(__file__).resolve().parent))
from test_quotient_gpu import make_columns  # noqa: E402

mzk = load()
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = mzk.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("k", [5, 9])
def test_compute_h_poly_matches_oracle(ctx, k):
    j = 5
    g = mzk.EvaluationDomain(ctx, j, k)
    o = O.Domain(j, k)
    n, E = g.n, g.extended_len
    cols = make_columns(300 + k, E, 3, 1, lookup_selector=6)
    cols["extended_omega"], cols["g_coset"] = o.get(2), o.get(3)
    host_desc = mzk.build_quotient_desc(cols, k, g.extended_k, lambda a: a.ctypes.data)
    odesc = O.QuotientDesc()
    ctypes.memmove(ctypes.byref(odesc), ctypes.byref(host_desc), ctypes.sizeof(odesc))
    h = o.extended_to_coeff(o.quotient_eval(odesc, True))
    qdeg = j - 1
    blinds = O.rand_fr(77 + k, qdeg - 1)
    limbs = []
    for i in range(qdeg):
        limb = np.concatenate([h[i * (n - 1):(i + 1) * (n - 1)],
                               (blinds[i] if i + 1 < qdeg else np.zeros(4, np.uint64)).reshape(1, 4)])
        if i > 0:
            limb[0] = O.fr_op("sub", limb[0], blinds[i - 1])
        limbs.append(limb)
    srs = O.gen_bases(0x5A5A + k, n)
    expect = [O.msm_best(limb, srs) for limb in limbs]

    bufs = {}

    def dev(a):
        if id(a) not in bufs:
            b = ctx.alloc(a.nbytes)
            b.upload(a)
            bufs[id(a)] = (b, a)
        return bufs[id(a)][0].ptr

    desc = mzk.build_quotient_desc(cols, k, g.extended_k, dev)
    d_srs = ctx.alloc(srs.nbytes)
    d_srs.upload(srs)
    d_limbs = ctx.alloc(qdeg * n * 32)
    got = g.compute_h_poly_device(desc, d_srs, n, blinds, d_limbs)
    assert np.array_equal(d_limbs.download((qdeg, n, 4)), np.stack(limbs))
    for i in range(qdeg):
        assert np.array_equal(mzk.affine(got[i]), expect[i]), i
