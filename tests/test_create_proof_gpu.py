"""create_proof on the B200 through the C ABI against the oracle's
restatement (oracle/plonk.py): device keygen gives the oracle's VK
commitments and transcript_repr; a proof of the single-proof configuration's
circuit (standard gate, copy cycles, range lookup) is byte-for-byte the
oracle's transcript at k = 5, 10 and 18, and the oracle's verifier accepts it
(with the G1 trapdoor check in place of the pairing) and rejects it once
tampered; many proofs of mixed k in one call equal each proof alone."""
import numpy as np
import pytest

from _plonk_setup import Circuit, mzk
from oracle import plonk as OP

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = mzk.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def k5(ctx):
    return Circuit(ctx, 5, seed=1)


def test_keygen_matches_oracle(k5):
    ok = k5.okey
    assert np.array_equal(k5.key.fixed_coms[:, :12], np.stack(ok.fixed_coms))
    assert np.array_equal(k5.key.perm_coms[:, :12], np.stack(ok.perm_coms))
    assert OP.to_int(k5.key.repr) == ok.repr
    assert k5.key.proof_len == 13 * 48 + 21 * 32
    assert k5.key.n_blinds == OP.blind_count(OP.config3_circuit(5))


@pytest.mark.parametrize("k", [5, 10])
def test_proof_bytes_equal_oracle_and_verify(ctx, k):
    c = Circuit(ctx, k, seed=k)
    for seed in (1, 2):
        bl = c.blinds(seed)
        proof = mzk.create_proofs(ctx, [(c.key, c.advice, bl)])[0]
        assert proof == c.oracle_proof(c.advice, bl)
        assert c.verify(proof)


def test_config3_k18_proof_equals_oracle_and_verifies(ctx):
    c = Circuit(ctx, 18, seed=18)
    bl = c.blinds(18)
    proof = mzk.create_proofs(ctx, [(c.key, c.advice, bl)], flags=mzk.PROVE_SELF_CHECK)[0]
    assert len(proof) == c.key.proof_len
    assert proof == c.oracle_proof(c.advice, bl)
    assert c.verify(proof)


def test_tampered_proof_is_rejected(k5):
    bl = k5.blinds(7)
    proof = mzk.create_proofs(k5.ctx, [(k5.key, k5.advice, bl)])[0]
    assert k5.verify(proof)
    for at in (5, 48 * 4 + 9, 13 * 48 - 1, len(proof) - 40):
        bad = bytearray(proof)
        bad[at] ^= 0x01
        assert not k5.verify(bytes(bad)), at


def test_batch_of_mixed_k_equals_each_alone(ctx, k5):
    c7 = Circuit(ctx, 7, seed=3, oracle=False)    # its own SRS buffer: proved in calls of its own
    jobs = [(k5.key, k5.advice, k5.blinds(1)), (c7.key, c7.advice, c7.blinds(2)), (k5.key, k5.advice, k5.blinds(3))]
    together = mzk.create_proofs(ctx, [jobs[0], jobs[2]])
    assert together[0] == mzk.create_proofs(ctx, [jobs[0]])[0]
    assert together[1] == mzk.create_proofs(ctx, [jobs[2]])[0]
    assert together[0] != together[1]
    # the plain form (every MSM its own call, no graphs) gives the same bytes
    plain = mzk.create_proofs(ctx, [jobs[0], jobs[2]], flags=mzk.PROVE_MSM_PER_CALL | mzk.PROVE_NO_GRAPHS)
    assert plain == together
    assert mzk.create_proofs(ctx, [jobs[1]])[0] == mzk.create_proofs(ctx, [jobs[1]], flags=mzk.PROVE_NO_GRAPHS)[0]


def test_mixed_k_over_one_srs(ctx):
    """Keys of k = 6 and k = 8 over one SRS buffer (each k's bases at its own
    offsets) prove in one call, and each proof equals its proof alone and the
    oracle's."""
    from oracle import oracle as O
    s = O.rand_fr(4242, 1)[0]
    sizes = {6: 1 << 6, 8: 1 << 8}
    total = sum(4 * n for n in sizes.values())
    buf = ctx.alloc(total * 96)
    offs, at = {}, 0
    for k, n in sizes.items():
        dom = mzk.EvaluationDomain(ctx, 5, k)
        p = buf.ptr + at * 96
        dom.srs_setup_device(s, p, p + n * 96, p + 2 * n * 96, p + 3 * n * 96)
        offs[k] = (at, at + n, at + 2 * n, at + 3 * n)
        at += 4 * n
        dom.close()
    cs = {}
    for k in sizes:
        d = mzk.SrsDesc(buf.ptr, total, *offs[k], 0, 0, 0)
        cs[k] = Circuit(ctx, k, seed=k + 30, srs=(buf, offs[k], d, s))
    jobs = [(cs[6].key, cs[6].advice, cs[6].blinds(1)), (cs[8].key, cs[8].advice, cs[8].blinds(2)),
            (cs[6].key, cs[6].advice, cs[6].blinds(3))]
    together = mzk.create_proofs(ctx, jobs)
    for j, pr in zip(jobs, together):
        assert pr == mzk.create_proofs(ctx, [j])[0]
    assert together[1] == cs[8].oracle_proof(cs[8].advice, jobs[1][2])
    assert cs[8].verify(together[1]) and cs[6].verify(together[0])


def test_device_advice_gives_the_same_proof(k5):
    ctx = k5.ctx
    bufs = []
    for col in k5.advice:
        b = ctx.alloc(col.nbytes)
        b.upload(col)
        bufs.append(b)
    bl = k5.blinds(4)
    assert mzk.create_proofs(ctx, [(k5.key, bufs, bl)])[0] == mzk.create_proofs(ctx, [(k5.key, k5.advice, bl)])[0]


def test_self_check_refuses_unsatisfied_witness(k5):
    ctx = k5.ctx
    bl = k5.blinds(5)
    assert mzk.create_proofs(ctx, [(k5.key, k5.advice, bl)], flags=mzk.PROVE_SELF_CHECK)
    bad = [a.copy() for a in k5.advice]
    bad[2][4] = OP.to_mont(OP.to_int(bad[2][4]) + 1)
    with pytest.raises(mzk.MzkError, match="does not satisfy"):
        mzk.create_proofs(ctx, [(k5.key, bad, bl)], flags=mzk.PROVE_SELF_CHECK)
    # without the check the proof is made, and the verifier rejects it
    assert not k5.verify(mzk.create_proofs(ctx, [(k5.key, bad, bl)])[0])


def test_lookup_input_outside_the_table_is_refused(k5):
    bad = [a.copy() for a in k5.advice]
    bad[0][1] = OP.to_mont(123456789)
    with pytest.raises(mzk.MzkError, match="not in the table"):
        mzk.create_proofs(k5.ctx, [(k5.key, bad, k5.blinds(6))])
    # the context stays usable
    assert k5.verify(mzk.create_proofs(k5.ctx, [(k5.key, k5.advice, k5.blinds(6))])[0])


def test_wrong_blind_count_is_refused(k5):
    with pytest.raises(mzk.MzkError):
        mzk.create_proofs(k5.ctx, [(k5.key, k5.advice, k5.blinds(1)[:-1])])


def test_device_generated_config3_instance_verifies(ctx):
    """The benchmark's device-generated instances (mzk_gen_config3_*): the
    fixed columns, copy cycles and a fresh witness satisfy the circuit (the
    self-check passes), and the proof is the oracle's transcript and verifies."""
    from oracle import oracle as O
    k = 10
    dom = mzk.EvaluationDomain(ctx, 5, k)
    n = dom.n
    s = O.rand_fr(99, 1)[0]
    buf = ctx.alloc(4 * n * 96)
    dom.srs_setup_device(s, buf.ptr, buf.ptr + n * 96, buf.ptr + 2 * n * 96, buf.ptr + 3 * n * 96)
    desc = mzk.SrsDesc(buf.ptr, 4 * n, 0, n, 2 * n, 3 * n, 0, 0, 0)
    inst = mzk.Config3Instance(ctx, dom, desc, seed=3, table_rows=300)
    wit, bl = inst.witness(5), inst.blinds(6)
    proof = mzk.create_proofs(ctx, [(inst.key, wit, bl)], flags=mzk.PROVE_SELF_CHECK)[0]
    host = buf.download((4 * n, 12))
    srs = {"g": host[:n], "lagrange": host[n:2 * n], "delta": host[2 * n:3 * n], "double_delta": host[3 * n:]}
    mapping = mzk.copy_cycles(n, n - 8, 3)[0]
    okey = OP.keygen(OP.config3_circuit(k), list(inst.fixed.download((7, n, 4))), mapping, srs, b"config-3 circuit")
    adv = list(wit[0].buf.download((3, n, 4)))
    assert OP.create_proof(okey, adv, [OP.to_int(v) for v in bl]) == proof
    assert OP.verify(okey, proof, OP.to_int(s))
    # a second fresh witness also satisfies the circuit
    assert mzk.create_proofs(ctx, [(inst.key, inst.witness(7), inst.blinds(8))], flags=mzk.PROVE_SELF_CHECK)


@pytest.mark.parametrize("k", [5, 8])
def test_generic_circuit_proof_equals_oracle(ctx, k):
    """A circuit of another shape (two gates as a flattened program reading
    a(wX), four permutation columns in two sets, the lookup): device keygen and
    create_proof give the oracle's transcript, it verifies, the self-check
    holds, and it proves through the proving service too."""
    c = Circuit(ctx, k, seed=k + 60, shape="generic")
    assert OP.to_int(c.key.repr) == c.okey.repr
    bl = c.blinds(3)
    proof = mzk.create_proofs(ctx, [(c.key, c.advice, bl)], flags=mzk.PROVE_SELF_CHECK)[0]
    assert proof == c.oracle_proof(c.advice, bl)
    assert c.verify(proof)
    srv = mzk.ProvingServer(ctx, max_batch=4)
    t = [srv.submit(c.key, c.advice, c.blinds(s)) for s in (3, 4)]
    outs = [srv.wait(x)[0] for x in t]
    srv.close()
    assert outs[0] == proof and c.verify(outs[1])
    bad = [a.copy() for a in c.advice]
    bad[3][2] = OP.to_mont(OP.to_int(bad[3][2]) + 1)
    with pytest.raises(mzk.MzkError, match="does not satisfy"):
        mzk.create_proofs(ctx, [(c.key, bad, bl)], flags=mzk.PROVE_SELF_CHECK)


@pytest.mark.parametrize("k", [5, 9])
def test_two_lookup_circuit_proof_equals_oracle(ctx, k):
    """Two lookups, the second (d into a table of squares) without a selector:
    per-lookup multiplicities, helpers and aggregators in the reference's
    transcript order, the quotient's lookup terms as helper programs.  The
    device transcript equals the oracle's and verifies, alone, in a batch and
    through the proving service; an input outside its table is refused."""
    c = Circuit(ctx, k, seed=k + 70, shape="generic2")
    assert len(c.circuit["lookups"]) == 2
    bl = c.blinds(5)
    proof = mzk.create_proofs(ctx, [(c.key, c.advice, bl)], flags=mzk.PROVE_SELF_CHECK)[0]
    assert proof == c.oracle_proof(c.advice, bl)
    assert c.verify(proof)
    both = mzk.create_proofs(ctx, [(c.key, c.advice, bl), (c.key, c.advice, c.blinds(6))])
    assert both[0] == proof and c.verify(both[1])
    srv = mzk.ProvingServer(ctx, max_batch=4)
    t = srv.submit(c.key, c.advice, c.blinds(7))
    assert c.verify(srv.wait(t)[0])
    srv.close()
    bad = [a.copy() for a in c.advice]
    bad[3][2] = OP.to_mont(OP.to_int(bad[3][2]) + 1)        # d no longer a square in the table
    with pytest.raises(mzk.MzkError, match="not in the table"):
        mzk.create_proofs(ctx, [(c.key, bad, bl)])


@pytest.mark.parametrize("k", [5, 9])
def test_instance_circuit_proof_equals_oracle(ctx, k):
    """An instance column (public inputs) read by a gate and copied into an
    advice column by the permutation: the values go into the transcript after
    the VK hash, the device transcript equals the oracle's and verifies with
    those public inputs, alone, in a batch and through the proving service;
    other public inputs fail the self-check, and more values than usable rows
    are refused."""
    c = Circuit(ctx, k, seed=k + 80, shape="instance")
    assert c.circuit["n_instance"] == 1 and c.instances is not None
    bl = c.blinds(5)
    proof = mzk.create_proofs(ctx, [(c.key, c.advice, bl, c.instances)], flags=mzk.PROVE_SELF_CHECK)[0]
    assert proof == c.oracle_proof(c.advice, bl)
    assert c.verify(proof)
    both = mzk.create_proofs(ctx, [(c.key, c.advice, bl, c.instances), (c.key, c.advice, c.blinds(6), c.instances)])
    assert both[0] == proof and c.verify(both[1])
    srv = mzk.ProvingServer(ctx, max_batch=4)
    t = srv.submit(c.key, c.advice, c.blinds(7), c.instances)
    assert c.verify(srv.wait(t)[0])
    srv.close()
    other = [c.instances[0].copy()]
    other[0][0] = OP.to_mont(OP.to_int(other[0][0]) + 1)
    assert not c.verify(proof, other)
    with pytest.raises(mzk.MzkError, match="does not satisfy"):
        mzk.create_proofs(ctx, [(c.key, c.advice, bl, other)], flags=mzk.PROVE_SELF_CHECK)
    with pytest.raises(mzk.MzkError, match="usable rows"):
        too_many = np.tile(c.instances[0][:1], (c.n - c.circuit["blinding_factors"], 1))   # usable rows + 1
        mzk.create_proofs(ctx, [(c.key, c.advice, bl, [too_many])])
    with pytest.raises(mzk.MzkError):
        mzk.create_proofs(ctx, [(c.key, c.advice, bl)])                # the instance column is missing


@pytest.mark.parametrize("k", [5, 9])
def test_trash_circuit_proof_equals_oracle(ctx, k):
    """A trashcan: its column (constraint expressions folded with the trash
    challenge, evaluated on the device over the Lagrange columns) committed
    after the trash challenge and before y, evaluated and opened at x; the
    lookup goes to the quotient as a helper program.  The device transcript
    equals the oracle's and verifies, alone, in a batch and through the
    proving service; a witness breaking a trashed constraint fails the
    self-check."""
    c = Circuit(ctx, k, seed=k + 90, shape="trash")
    assert len(c.circuit["trashcans"]) == 1
    bl = c.blinds(5)
    proof = mzk.create_proofs(ctx, [(c.key, c.advice, bl)], flags=mzk.PROVE_SELF_CHECK)[0]
    assert proof == c.oracle_proof(c.advice, bl)
    assert c.verify(proof)
    both = mzk.create_proofs(ctx, [(c.key, c.advice, bl), (c.key, c.advice, c.blinds(6))])
    assert both[0] == proof and c.verify(both[1])
    srv = mzk.ProvingServer(ctx, max_batch=4)
    t = srv.submit(c.key, c.advice, c.blinds(7))
    assert c.verify(srv.wait(t)[0])
    srv.close()
    assert replay(c.key, proof) == proof                    # the layout lists the trash commitment and evaluation
    bad = [a.copy() for a in c.advice]
    bad[3][1] = OP.to_mont(OP.to_int(bad[3][1]) + 1)          # d != a^2 on a row where q3 is set
    with pytest.raises(mzk.MzkError, match="does not satisfy"):
        mzk.create_proofs(ctx, [(c.key, bad, bl)], flags=mzk.PROVE_SELF_CHECK)


@pytest.mark.parametrize("k", [5, 9])
def test_simple_selector_proof_equals_oracle(ctx, k):
    """A simple selector (q3 of the second gate polynomial): its evaluation is
    one in the identities, it is neither written nor opened, and its fixed
    polynomial enters the linearization scaled by the gate polynomial at x.
    The device transcript equals the oracle's and verifies, in a batch and
    through the proving service, and replays from the layout; a witness
    breaking the selected gate fails the self-check."""
    c = Circuit(ctx, k, seed=k + 100, shape="selector")
    assert c.circuit["gate_polys"][1][1] == 2
    bl = c.blinds(5)
    proof = mzk.create_proofs(ctx, [(c.key, c.advice, bl)], flags=mzk.PROVE_SELF_CHECK)[0]
    assert proof == c.oracle_proof(c.advice, bl)
    assert c.verify(proof)
    assert replay(c.key, proof) == proof
    both = mzk.create_proofs(ctx, [(c.key, c.advice, bl), (c.key, c.advice, c.blinds(6))])
    assert both[0] == proof and c.verify(both[1])
    srv = mzk.ProvingServer(ctx, max_batch=4)
    t = srv.submit(c.key, c.advice, c.blinds(7))
    assert c.verify(srv.wait(t)[0])
    srv.close()
    bad = [a.copy() for a in c.advice]
    bad[3][1] = OP.to_mont(OP.to_int(bad[3][1]) + 1)          # d != a^2 on a selected row
    with pytest.raises(mzk.MzkError, match="does not satisfy"):
        mzk.create_proofs(ctx, [(c.key, bad, bl)], flags=mzk.PROVE_SELF_CHECK)


@pytest.mark.parametrize("k", [5, 9])
def test_tuple_lookup_proof_equals_oracle(ctx, k):
    """A lookup of the tuple (a, d) into (table, squares): multiplicities by
    matching tuples against the key's tuple index, the logup helper over the
    theta-compressed input and table, the quotient's lookup term as a tuple
    helper program.  The device transcript equals the oracle's and verifies,
    in a batch and through the proving service; a tuple outside the table is
    refused."""
    c = Circuit(ctx, k, seed=k + 110, shape="tuple")
    bl = c.blinds(5)
    proof = mzk.create_proofs(ctx, [(c.key, c.advice, bl)], flags=mzk.PROVE_SELF_CHECK)[0]
    assert proof == c.oracle_proof(c.advice, bl)
    assert c.verify(proof)
    both = mzk.create_proofs(ctx, [(c.key, c.advice, bl), (c.key, c.advice, c.blinds(6))])
    assert both[0] == proof and c.verify(both[1])
    srv = mzk.ProvingServer(ctx, max_batch=4)
    t = srv.submit(c.key, c.advice, c.blinds(7))
    assert c.verify(srv.wait(t)[0])
    srv.close()
    bad = [a.copy() for a in c.advice]
    bad[3][1] = OP.to_mont(OP.to_int(bad[3][1]) + 1)          # (a, d) no longer a row of the table
    with pytest.raises(mzk.MzkError, match="not in the table"):
        mzk.create_proofs(ctx, [(c.key, bad, bl)])


@pytest.mark.parametrize("k", [5, 9])
def test_parallel_lookup_proof_equals_oracle(ctx, k):
    """Lookups with parallel inputs: five columns into one table (helper
    chunks of four and one at degree 5, committed, evaluated and opened per
    chunk, one quotient helper program each, with the partial products) and
    two theta-compressed tuples into (table, squares) in one chunk.  The
    device transcript equals the oracle's and verifies, in a batch and
    through the proving service; an input outside its table is refused."""
    c = Circuit(ctx, k, seed=k + 120, shape="parallel")
    assert c.key.proof_len == len(c.oracle_proof(c.advice, c.blinds(4)))
    bl = c.blinds(5)
    proof = mzk.create_proofs(ctx, [(c.key, c.advice, bl)], flags=mzk.PROVE_SELF_CHECK)[0]
    assert proof == c.oracle_proof(c.advice, bl)
    assert c.verify(proof)
    both = mzk.create_proofs(ctx, [(c.key, c.advice, bl), (c.key, c.advice, c.blinds(6))])
    assert both[0] == proof and c.verify(both[1])
    srv = mzk.ProvingServer(ctx, max_batch=4)
    t = srv.submit(c.key, c.advice, c.blinds(7))
    assert c.verify(srv.wait(t)[0])
    srv.close()
    bad = [a.copy() for a in c.advice]
    bad[5][2] = OP.to_mont((1 << 16) + 5)                      # f outside the table on a selected row
    with pytest.raises(mzk.MzkError, match="not in the table"):
        mzk.create_proofs(ctx, [(c.key, bad, bl)])


@pytest.mark.parametrize("k", [6, 9])
def test_five_lookups_and_five_trashcans_equal_oracle(ctx, k):
    """Five lookups and five trashcans (more than a key of four of each
    takes): the device transcript equals the oracle's and verifies, alone
    and in a batch."""
    c = Circuit(ctx, k, seed=k + 160, shape="many")
    assert c.key.proof_len == len(c.oracle_proof(c.advice, c.blinds(4)))
    bl = c.blinds(5)
    proof = mzk.create_proofs(ctx, [(c.key, c.advice, bl)], flags=mzk.PROVE_SELF_CHECK)[0]
    assert proof == c.oracle_proof(c.advice, bl)
    assert c.verify(proof)
    both = mzk.create_proofs(ctx, [(c.key, c.advice, c.blinds(6)), (c.key, c.advice, bl)])
    assert both[1] == proof and c.verify(both[0])


@pytest.mark.parametrize("k", [5, 9])
def test_expression_lookup_inputs_equal_oracle(ctx, k):
    """Lookup inputs that are expressions (a(wX) and d - a^2 + a into the
    table, the tuple (a, a * a) into (table, squares)): each evaluated over
    the Lagrange rows for the multiplicities and helpers and over the
    extended coset for the quotient, and at x for the identities.  The device
    transcript equals the oracle's and verifies, in a batch and through the
    proving service; an input outside the table is refused; an input
    expression whose degree leaves no room for a helper constraint is refused
    by keygen."""
    c = Circuit(ctx, k, seed=k + 150, shape="expr")
    assert c.key.proof_len == len(c.oracle_proof(c.advice, c.blinds(4)))
    bl = c.blinds(5)
    proof = mzk.create_proofs(ctx, [(c.key, c.advice, bl)], flags=mzk.PROVE_SELF_CHECK)[0]
    assert proof == c.oracle_proof(c.advice, bl)
    assert c.verify(proof)
    both = mzk.create_proofs(ctx, [(c.key, c.advice, bl), (c.key, c.advice, c.blinds(6))])
    assert both[0] == proof and c.verify(both[1])
    srv = mzk.ProvingServer(ctx, max_batch=4)
    t = srv.submit(c.key, c.advice, c.blinds(7))
    assert c.verify(srv.wait(t)[0])
    srv.close()
    bad = [a.copy() for a in c.advice]
    bad[0][3] = OP.to_mont((1 << 16) + 9)                       # a(wX) on row 2 outside the table
    with pytest.raises(mzk.MzkError, match="not in the table"):
        mzk.create_proofs(ctx, [(c.key, bad, bl)])
    if k == 5:
        deep = OP.expr_circuit(k)
        a5 = OP._expr_program([0], [(1, 0, 0, 7)], [(3, 8, 7, 0, 0), (3, 9, 8, 0, 0), (2, 10, 9, 7, 0)], 11, 10)
        deep["lookups"] = [{"input": a5, "table": 4, "selector": 3}]   # a^5: degree 5 > next_pow2(5 - 1)
        deep["blinding_factors"] = OP.blinding_factors(c.circuit)
        with pytest.raises(mzk.MzkError, match="exceed cs.degree"):
            mzk.PlonkKey(ctx, c.dom, deep, c.desc, c.fixed, c.mapping, b"deep")


@pytest.mark.parametrize("shape", ["nolookup", "bare"])
@pytest.mark.parametrize("k", [5, 9])
def test_circuits_without_lookup_or_permutation_equal_oracle(ctx, k, shape):
    """A circuit without lookups, and one without lookups and permutation
    (no z, m, h or Z; a key without permutation polynomials): the device
    transcript equals the oracle's and verifies, alone, in a batch with the
    other shape's proofs and through the proving service."""
    c = Circuit(ctx, k, seed=k + 130, shape=shape)
    assert c.key.proof_len == len(c.oracle_proof(c.advice, c.blinds(4)))
    bl = c.blinds(5)
    proof = mzk.create_proofs(ctx, [(c.key, c.advice, bl)], flags=mzk.PROVE_SELF_CHECK)[0]
    assert proof == c.oracle_proof(c.advice, bl)
    assert c.verify(proof)
    other = Circuit(ctx, k, seed=k + 140, shape="generic", srs=(c.srs_buf, c.offs, c.desc, c.s))
    mixed = mzk.create_proofs(ctx, [(c.key, c.advice, bl), (other.key, other.advice, other.blinds(6))])
    assert mixed[0] == proof and other.verify(mixed[1])
    srv = mzk.ProvingServer(ctx, max_batch=4)
    t = srv.submit(c.key, c.advice, c.blinds(7))
    assert c.verify(srv.wait(t)[0])
    srv.close()


def test_key_files_equal_oracle_and_read_back(ctx, k5):
    """VerifyingKey / ProvingKey files in the three SerdeFormats equal the
    oracle's bytes; a key read from a PK file has the same transcript_repr and
    gives the same proofs; damaged files are refused."""
    key, ok = k5.key, k5.okey
    for fmt, processed in ((mzk.SERDE_PROCESSED, True), (mzk.SERDE_RAW, False), (mzk.SERDE_RAW_UNCHECKED, False)):
        assert key.vk_bytes(fmt) == OP.vk_bytes(ok, processed), fmt
        pk = key.pk_bytes(fmt)
        assert pk == OP.pk_bytes(ok, processed), fmt
        back = mzk.PlonkKey(ctx, k5.dom, k5.circuit, k5.desc, pk_bytes=pk, pk_format=fmt,
                            pinned=b"config-3 circuit: standard gate, copy cycles, range lookup")
        assert np.array_equal(back.repr, key.repr) and back.pk_bytes(fmt) == pk
        bl = k5.blinds(11)
        assert mzk.create_proofs(ctx, [(back, k5.advice, bl)]) == mzk.create_proofs(ctx, [(key, k5.advice, bl)])
        back.close()
    pk = key.pk_bytes(mzk.SERDE_RAW)
    bad_cases = {
        "version": b"\x02" + pk[1:],
        "truncated": pk[:-1],
        "trailing": pk + b"\x00",
        "not below r": pk[:-32] + b"\xff" * 32,
        "not on the curve": pk[:6] + pk[6:54] + bytes(47) + b"\x05" + pk[102:],
    }
    for name, data in bad_cases.items():
        with pytest.raises(mzk.MzkError):
            mzk.PlonkKey(ctx, k5.dom, k5.circuit, k5.desc, pk_bytes=data, pk_format=mzk.SERDE_RAW)
        assert name


def replay(key, proof):
    """The proof's transcript rebuilt from the key's transcript layout by a
    separate transcript object; returns its final bytes."""
    from oracle import oracle as O
    t, pos = mzk.Transcript(), 0
    for op in key.transcript_layout():
        if op == 0:
            t.common_fr(key.repr)
        elif op == 1:
            st, aff = O.g1_decompress(proof[pos:pos + 48])
            p18 = np.zeros(18, np.uint64)
            if np.any(aff):
                p18[:12], p18[12:] = aff, O.fp_const(0)
            t.write_point(p18)
            pos += 48
        elif op == 2:
            t.write_fr(OP.to_mont(int.from_bytes(proof[pos:pos + 32], "little")))
            pos += 32
        else:
            t.squeeze_challenge()
    assert pos == len(proof)
    return t.finalize()


def test_transcript_layout_replays_the_proof(k5):
    """A caller with its own transcript object replays a proof from the key's
    transcript layout: the same absorbs and squeezes rebuild the same proof
    bytes."""
    proof = mzk.create_proofs(k5.ctx, [(k5.key, k5.advice, k5.blinds(12))])[0]
    assert replay(k5.key, proof) == proof
