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


def test_device_derives_z_h_Z(ctx):
    """Jobs that leave z, h and Z null: the device derives them (permutation
    and logup arguments) and the commitments equal those of the same proof
    with the oracle's z, h and Z passed in."""
    from oracle import oracle as O
    st = Setup(ctx, 9, seed=9)
    n, bf = st.n, 7
    for seed in (21, 22):
        job, w, ch, blinds = st.job(seed)
        pblinds = O.rand_fr(seed * 50 + 40, bf)
        lblinds = O.rand_fr(seed * 50 + 41, bf)
        for i in range(bf):
            job.perm_blinds[i][:] = [int(v) for v in pblinds[i]]
            job.lookup_blinds[i][:] = [int(v) for v in lblinds[i]]
        z = O.permutation_z([w["a"], w["b"], w["c"]], st.sigma_lag, 3, 9, st.o.get(0), ch["beta"], ch["gamma"], bf,
                            pblinds.reshape(1, bf, 4))[0]
        (h,), Z = O.logup([[w["a"]]], st.table_lag, st.sel_lag, w["m"], ch["beta"], bf, lblinds)
        given = mzk.ProofJob()
        ctypes_copy(given, job)
        given.perm_z, given.lookup_h, given.lookup_Z = st.dev(z), st.dev(h), st.dev(Z)
        job.perm_z = job.lookup_h = job.lookup_Z = None
        derived = st.g.prove_core_device(st.pk, [job])[0]
        expect = st.g.prove_core_device(st.pk, [given])[0]
        assert np.array_equal(derived, expect)
        # and z alone derived, h and Z given
        mixed = mzk.ProofJob()
        ctypes_copy(mixed, given)
        mixed.perm_z = None
        assert np.array_equal(st.g.prove_core_device(st.pk, [mixed])[0], expect)


def ctypes_copy(dst, src):
    import ctypes
    ctypes.memmove(ctypes.byref(dst), ctypes.byref(src), ctypes.sizeof(src))


def test_ntt_sequence_graph_replays_equal_launches(ctx):
    """Each proof's NTT sequence is captured into a CUDA graph once per key
    and replayed afterwards: the commitments equal those of the kernel-by-
    kernel launches, replays happen on repeated calls, and destroying a domain
    drops the graphs (a new domain at the same address is captured afresh)."""
    c = mzk.Context(0)
    try:
        st = Setup(c, 8, seed=31)
        jobs = [st.job(s)[0] for s in (41, 42)]
        eager = st.g.prove_core_device(st.pk, jobs, graphs=False)
        assert c.graph_stats() == (0, 0)
        first = st.g.prove_core_device(st.pk, jobs)
        caps, reps = c.graph_stats()
        assert caps == 2 and reps == 0                 # one graph per proof slot of the wave
        again = st.g.prove_core_device(st.pk, jobs)
        assert c.graph_stats() == (2, 2)
        assert np.array_equal(first, eager) and np.array_equal(again, eager)
        st2 = Setup(c, 8, seed=31)                     # same circuit, fresh domain and key buffers
        st.g.close()
        assert np.array_equal(st2.g.prove_core_device(st2.pk, jobs), eager)
        assert c.graph_stats()[0] >= 3                 # recaptured after the domain went away
    finally:
        c.close()


def test_graph_captured_before_its_pass_twiddle_tables_exist():
    """A transform captured into a graph while the twiddle tables of its
    passes do not exist yet (the NTT split changed after the domain was made,
    and a table is never built during a capture) forms its inter-pass
    twiddles from the small root tables instead: the captured proof's
    commitments equal the eager launches', which build the tables."""
    c = mzk.Context(0)
    try:
        st = Setup(c, 12, seed=37)
        for lg in (st.g.k, st.g.extended_k):
            c.set_tuned(c.TUNE_NTT_SPLIT, lg, 3)        # largest passes last: new pass shapes
        jobs = [st.job(s)[0] for s in (43, 44)]
        captured = st.g.prove_core_device(st.pk, jobs)
        assert c.graph_stats()[0] == 2
        eager = st.g.prove_core_device(st.pk, jobs, graphs=False)
        assert np.array_equal(captured, eager)
        assert np.array_equal(st.g.prove_core_device(st.pk, jobs), eager)   # replayed
    finally:
        c.close()
