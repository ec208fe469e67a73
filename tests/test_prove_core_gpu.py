"""Device part of create_proof (witness commitments in their bases, the seven
lagrange_to_coeff / coeff_to_extended, compute_h_poly and the limb
commitments) against the oracle doing the same steps, for several proofs in
one call; and a batch equals its proofs run alone."""
import numpy as np
import pytest

from _proof_setup import Setup, mzk
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = mzk.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("k", [5, 8])
def test_prove_core_matches_oracle(ctx, k):
    st = Setup(ctx, k, seed=k)
    jobs = [st.job(s) for s in (1, 2, 3)]
    got = st.g.prove_core_device(st.pk, [j for j, _, _, _ in jobs])
    for pi, (_, w, ch, blinds) in enumerate(jobs):
        expect = st.oracle(w, ch, blinds)
        for ci, name in enumerate(mzk.PROOF_CORE_COMMITMENTS):
            assert np.array_equal(mzk.affine(got[pi, ci]), expect[ci]), (pi, name)


def test_prove_core_batch_equals_single(ctx):
    st = Setup(ctx, 10, seed=4)
    jobs = [st.job(s)[0] for s in (5, 6, 7, 8)]
    together = st.g.prove_core_device(st.pk, jobs)
    for i, j in enumerate(jobs):
        assert np.array_equal(st.g.prove_core_device(st.pk, [j])[0], together[i])
    # the plain form (every MSM its own call) gives the same commitments
    assert np.array_equal(st.g.prove_core_device(st.pk, jobs[:2], per_call=True), together[:2])
