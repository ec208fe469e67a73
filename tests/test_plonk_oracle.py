"""The oracle's create_proof and verifier (oracle/plonk.py) on the
single-proof configuration's circuit: honest proofs are accepted, and the
verifier rejects every kind of wrong proof it must reject (tampered
commitments and evaluations, truncated or extended proofs, a wrong trapdoor,
witnesses that break the gate or a copy constraint).  CPU only."""
import numpy as np
import pytest

from oracle import oracle as O
from oracle import plonk as OP


def setup(k, seed, pinned=b"config-3 circuit"):
    c = OP.config3_circuit(k)
    fixed, mapping, adv = OP.config3_instance(k, seed)
    s = O.rand_fr(1000 + seed, 1)[0]
    g, lag, dl, ddl = O.srs_setup(s, k)
    srs = {"g": g, "lagrange": lag, "delta": dl, "double_delta": ddl}
    key = OP.keygen(c, fixed, mapping, srs, pinned)
    return c, key, adv, OP.to_int(s), mapping


def blinds(c, seed):
    return [OP.to_int(v) for v in O.rand_fr(2000 + seed, OP.blind_count(c))]


@pytest.fixture(scope="module")
def k5():
    c, key, adv, s, mapping = setup(5, 1)
    proof = OP.create_proof(key, adv, blinds(c, 1))
    return c, key, adv, s, mapping, proof


def test_shape_constants(k5):
    c, key, _, _, _, proof = k5
    assert OP.blinding_factors(c) == 7 and key.qdeg == 4 and key.dom.extended_k == 7
    # 13 commitments (a, b, c, m, z, h, Z, 4 limbs, f, pi) and 21 scalars
    assert len(proof) == 13 * 48 + 21 * 32


def test_honest_proofs_verify(k5):
    _, key, _, s, _, proof = k5
    assert OP.verify(key, proof, s)
    c, key7, adv7, s7, _ = setup(7, 2)
    assert OP.verify(key7, OP.create_proof(key7, adv7, blinds(c, 2)), s7)


def test_proofs_are_deterministic_in_the_blinds(k5):
    c, key, adv, _, _, proof = k5
    assert OP.create_proof(key, adv, blinds(c, 1)) == proof
    assert OP.create_proof(key, adv, blinds(c, 3)) != proof


def test_tampered_proofs_are_rejected(k5):
    _, key, _, s, _, proof = k5
    gen = bytes(O.g1_compress(O.g1_generator()))
    for at in (0, 48 * 3, 48 * 7, 48 * 10):            # a, m, h, a quotient limb
        bad = proof[:at] + gen + proof[at + 48:]
        assert not OP.verify(key, bad, s), at
    pts = 11 * 48
    for i in range(0, 19):                              # every evaluation before the multi-open
        at = pts + 32 * i
        v = int.from_bytes(proof[at:at + 32], "little")
        bad = proof[:at] + ((v + 1) % OP.R).to_bytes(32, "little") + proof[at + 32:]
        assert not OP.verify(key, bad, s), i
    assert not OP.verify(key, proof[:-1], s)
    assert not OP.verify(key, proof + b"\x00", s)
    assert not OP.verify(key, proof, s + 1)


def test_unsatisfied_witnesses_are_rejected(k5):
    c, key, adv, s, mapping, _ = k5
    bad = [a.copy() for a in adv]
    bad[2][3] = OP.to_mont(OP.to_int(bad[2][3]) + 1)    # the gate fails on row 3
    assert not OP.verify(key, OP.create_proof(key, bad, blinds(c, 1)), s)
    # a copy constraint fails: a cell of a cycle changes (a b-cell, so the lookup still holds),
    # its row's c is solved again so the gate still holds
    cyc = [(cc, r) for cc in range(2) for r in range(key.u) if tuple(mapping[cc, r]) != (cc, r)]
    cc, r = next((cc, r) for cc, r in cyc if cc == 1)
    bad = [a.copy() for a in adv]
    fixed = key.fixed_values
    bad[1][r] = OP.to_mont(OP.to_int(bad[1][r]) + 5)
    ql, qr, qm, qo, qcst = (OP.to_int(fixed[i][r]) for i in range(5))
    a, b = OP.to_int(bad[0][r]), OP.to_int(bad[1][r])
    bad[2][r] = OP.to_mont(-(ql * a + qr * b + qm * a * b + qcst) * OP.inv(qo))
    assert not OP.verify(key, OP.create_proof(key, bad, blinds(c, 1)), s)


def test_lookup_input_outside_the_table_is_refused(k5):
    c, key, adv, _, _, _ = k5
    bad = [a.copy() for a in adv]
    bad[0][2] = OP.to_mont(10 ** 9)
    with pytest.raises(ValueError):
        OP.create_proof(key, bad, blinds(c, 1))


def test_intermediate_sets_follow_first_appearance():
    q = [("a", 1), ("b", 1), ("z", 1), ("z", 7), ("b", 9), ("c", 1), ("Z", 1), ("Z", 7)]
    labels, sets, _ = OP.intermediate_sets(q)
    assert [lb for lb, _, _ in labels] == ["a", "b", "z", "c", "Z"]
    assert sets == [[1], [1, 9], [1, 7]]
    assert [si for _, si, _ in labels] == [0, 1, 2, 0, 2]
    with pytest.raises(ValueError):
        OP.intermediate_sets([("a", 1), ("a", 1)])


@pytest.mark.parametrize("k", [5, 6])
def test_quotient_work_count(k):
    """The quotient of the single-proof configuration costs 37 Fr
    multiplications per extended row (gate 5, permutation set and boundary
    terms with the y-Horner steps, the lookup terms, the division by t(X)),
    plus one for beta * g_coset: the work figure of the quotient's roofline,
    counted on the oracle's restatement of evaluate_numerator with omega^idx
    stepped as the reference steps it."""
    c, key, _, _, _ = setup(k, 3)
    E = key.dom.extended_len
    cols = [O.rand_fr(70 + i, E) for i in range(7)]
    _, count = O.count_fr_muls(OP.quotient, key, cols[:3], [cols[3]], [cols[4]], [cols[5]], [cols[6]], 1, 2, 3, 4,
                               threads=1)
    assert count == 37 * E + 1


def test_two_lookup_circuit_proofs_verify():
    """Two lookups, the second without a selector: multiplicities, helpers and
    aggregators committed, evaluated and opened lookup by lookup; the
    quotient takes the lookups as helper programs.  A proof verifies, a
    tampered one does not, and an input outside its table is refused."""
    k = 5
    c = OP.generic2_circuit(k)
    fixed, mapping, adv = OP.generic2_instance(k, 11)
    s = O.rand_fr(58, 1)[0]
    g, lag, dl, ddl = O.srs_setup(s, k)
    key = OP.keygen(c, fixed, mapping, {"g": g, "lagrange": lag, "delta": dl, "double_delta": ddl}, b"generic2")
    assert len(c["lookups"]) == 2 and key.bf == OP.blinding_factors(c)
    bl = [OP.to_int(v) for v in O.rand_fr(68, OP.blind_count(c))]
    proof = OP.create_proof(key, adv, bl)
    A, L, S, qdeg = 4, 2, 2, 4
    points = A + L + S + 2 * L + qdeg + 2                      # advice, m, z, (h, Z), limbs, f, pi
    scalars_before_q = len(c["advice_queries"]) + len(c["fixed_queries"]) + 4 + (3 * S - 1) + 4 * L
    assert (len(proof) - 48 * points - 32 * scalars_before_q) // 32 in range(2, 8)   # the q evaluations
    assert OP.verify(key, proof, OP.to_int(s))
    bad = bytearray(proof)
    bad[4 * 48 + 48 + 5] ^= 1                                  # the second multiplicity commitment
    assert not OP.verify(key, bytes(bad), OP.to_int(s))
    wrong = [a.copy() for a in adv]
    wrong[3][2] = OP.to_mont(OP.to_int(wrong[3][2]) + 1)       # d no longer a square in the table
    with pytest.raises(ValueError):
        OP.create_proof(key, wrong, bl)


def test_instance_circuit_proofs_verify():
    """An instance column (public inputs): its values absorbed after the VK
    hash (compute_instances), read by a gate and copied into c by the
    permutation; the verifier evaluates it from the values.  The proof
    verifies with its public inputs and not with others; too many values are
    refused (Error::InstanceTooLarge)."""
    k = 5
    c = OP.instance_circuit(k)
    fixed, mapping, adv, inst = OP.instance_instance(k, 12)
    s = O.rand_fr(59, 1)[0]
    g, lag, dl, ddl = O.srs_setup(s, k)
    key = OP.keygen(c, fixed, mapping, {"g": g, "lagrange": lag, "delta": dl, "double_delta": ddl}, b"instance")
    assert OP.n_perm_sets(c) == 2 and len(c["perm_cols"]) == 5
    bl = [OP.to_int(v) for v in O.rand_fr(69, OP.blind_count(c))]
    proof = OP.create_proof(key, adv, bl, inst)
    assert OP.verify(key, proof, OP.to_int(s), inst)
    other = [inst[0].copy()]
    other[0][1] = OP.to_mont(OP.to_int(other[0][1]) + 1)
    assert not OP.verify(key, proof, OP.to_int(s), other)
    # a witness whose c disagrees with the public input fails the gate and the copy
    assert not OP.verify(key, OP.create_proof(key, adv, bl, other), OP.to_int(s), other)
    with pytest.raises(ValueError):
        OP.create_proof(key, adv, bl, [np.tile(O.fr_const(0), (key.u + 1, 1))])


def test_trash_circuit_proofs_verify():
    """A trashcan: its column (the constraint expressions folded with the
    trash challenge) committed after the trash challenge, evaluated and
    opened at x, its term compressed - (1 - q) trash in the identities; the
    lookup then goes to the quotient as a helper program.  The proof
    verifies; a witness breaking a trashed constraint on a selected row does
    not."""
    k = 5
    c = OP.trash_circuit(k)
    fixed, mapping, adv = OP.trash_instance(k, 13)
    s = O.rand_fr(57, 1)[0]
    g, lag, dl, ddl = O.srs_setup(s, k)
    key = OP.keygen(c, fixed, mapping, {"g": g, "lagrange": lag, "delta": dl, "double_delta": ddl}, b"trash")
    assert key.bf == OP.blinding_factors(OP.generic_circuit(k)) + 1
    bl = [OP.to_int(v) for v in O.rand_fr(67, OP.blind_count(c))]
    proof = OP.create_proof(key, adv, bl)
    assert OP.verify(key, proof, OP.to_int(s))
    bad = [a.copy() for a in adv]
    bad[3][1] = OP.to_mont(OP.to_int(bad[3][1]) + 1)          # d != a^2 on a row where q3 is set
    assert not OP.verify(key, OP.create_proof(key, bad, bl), OP.to_int(s))


def test_simple_selector_proofs_verify():
    """A simple selector: q3's evaluation is one in the identities, absent from
    the transcript and the openings, and its fixed polynomial enters the
    linearization scaled by d(x) - a(x)^2.  The proof verifies and is one
    scalar shorter than the same circuit's without the selector; a witness
    breaking the selected gate does not verify."""
    k = 5
    fixed, mapping, adv = OP.selector_instance(k, 14)
    s = O.rand_fr(56, 1)[0]
    g, lag, dl, ddl = O.srs_setup(s, k)
    srs = {"g": g, "lagrange": lag, "delta": dl, "double_delta": ddl}
    key = OP.keygen(OP.selector_circuit(k), fixed, mapping, srs, b"selector")
    c = OP.selector_circuit(k)
    bl = [OP.to_int(v) for v in O.rand_fr(66, OP.blind_count(c))]
    proof = OP.create_proof(key, adv, bl)
    assert OP.verify(key, proof, OP.to_int(s))
    plain = OP.keygen(OP.generic_circuit(k), fixed, mapping, srs, b"selector")
    assert len(OP.create_proof(plain, adv, bl)) - len(proof) in (32, 32 + 32)  # one evaluation (and maybe a q)
    bad = [a.copy() for a in adv]
    bad[3][1] = OP.to_mont(OP.to_int(bad[3][1]) + 1)          # d != a^2 on a selected row
    assert not OP.verify(key, OP.create_proof(key, bad, bl), OP.to_int(s))


def test_tuple_lookup_proofs_verify():
    """A lookup of the tuple (a, d) into (table, squares), compressed with
    theta on both sides: the proof verifies; a witness whose tuple is not a
    table row (d != a^2 on a selected row) is refused by the prover."""
    k = 5
    c = OP.tuple_circuit(k)
    fixed, mapping, adv = OP.tuple_instance(k, 15)
    s = O.rand_fr(55, 1)[0]
    g, lag, dl, ddl = O.srs_setup(s, k)
    key = OP.keygen(c, fixed, mapping, {"g": g, "lagrange": lag, "delta": dl, "double_delta": ddl}, b"tuple")
    bl = [OP.to_int(v) for v in O.rand_fr(65, OP.blind_count(c))]
    proof = OP.create_proof(key, adv, bl)
    assert OP.verify(key, proof, OP.to_int(s))
    bad = [a.copy() for a in adv]
    bad[3][1] = OP.to_mont(OP.to_int(bad[3][1]) + 1)
    with pytest.raises(ValueError):
        OP.create_proof(key, bad, bl)


def test_parallel_lookup_proofs_verify():
    """Lookups with parallel inputs (five columns into one table: helper
    chunks of four and one at degree 5; two theta-compressed tuples): the
    blinding factors count the three helpers, the proof verifies, a wrong
    helper evaluation or an input value outside the table is refused."""
    k = 5
    c = OP.parallel_circuit(k)
    assert [len(OP.lookup_chunks(c, lk)) for lk in c["lookups"]] == [2, 1]
    assert [len(ch) for ch in OP.lookup_chunks(c, c["lookups"][0])] == [4, 1]
    assert OP.blinding_factors(c) == 3 + 3 + 3
    fixed, mapping, adv = OP.parallel_instance(k, 21)
    s = O.rand_fr(56, 1)[0]
    g, lag, dl, ddl = O.srs_setup(s, k)
    key = OP.keygen(c, fixed, mapping, {"g": g, "lagrange": lag, "delta": dl, "double_delta": ddl}, b"parallel")
    bl = [OP.to_int(v) for v in O.rand_fr(66, OP.blind_count(c))]
    proof = OP.create_proof(key, adv, bl)
    assert OP.verify(key, proof, OP.to_int(s))
    # the evaluations start after 7 advice, 2 multiplicity, 2 permutation,
    # 3 helper, 2 aggregator and 4 quotient-limb points; the lookups' come
    # after 8 advice, 7 fixed, 4 permutation-column and 5 permutation-set
    # evaluations as m, h0, h1, Z, Z(wx) of the first lookup: flip the low
    # bit of its second helper's
    at = 20 * 48 + (8 + 7 + 4 + 5 + 2) * 32
    bad = bytearray(proof)
    bad[at] ^= 1
    assert not OP.verify(key, bytes(bad), OP.to_int(s))
    worse = [a.copy() for a in adv]
    worse[5][2] = OP.to_mont((1 << 16) + 5)                     # f outside the table on a selected row
    with pytest.raises(ValueError):
        OP.create_proof(key, worse, bl)


def test_five_lookups_and_five_trashcans_verify():
    """Five lookups (with and without selectors, a tuple) and five
    trashcans: the proof verifies and a tampered evaluation is rejected."""
    k = 6
    c = OP.many_circuit(k)
    assert OP.blinding_factors(c) == 3 + 5 + 5 + 3
    fixed, mapping, adv = OP.many_instance(k, 25)
    s = O.rand_fr(59, 1)[0]
    g, lag, dl, ddl = O.srs_setup(s, k)
    key = OP.keygen(c, fixed, mapping, {"g": g, "lagrange": lag, "delta": dl, "double_delta": ddl}, b"many")
    bl = [OP.to_int(v) for v in O.rand_fr(69, OP.blind_count(c))]
    proof = OP.create_proof(key, adv, bl)
    assert OP.verify(key, proof, OP.to_int(s))
    bad = bytearray(proof)
    bad[-48 * 2 - 32 * 3] ^= 1                                   # a q evaluation
    assert not OP.verify(key, bytes(bad), OP.to_int(s))


def test_expression_lookup_inputs_verify():
    """Lookup inputs that are expressions (a(wX), d - a^2 + a, a * a): their
    degree sets the inputs per helper (two at degree 5 for a degree-2 input),
    the proof verifies, and a witness whose rotated input leaves the table
    on a selected row is refused by the prover."""
    k = 5
    c = OP.expr_circuit(k)
    assert [OP.lookup_per_helper(c, lk) for lk in c["lookups"]] == [2, 2]
    assert [len(OP.lookup_chunks(c, lk)) for lk in c["lookups"]] == [1, 1]
    assert len(OP.lookup_exprs(c)) == 3 and OP.blinding_factors(c) == 3 + 2 + 3
    fixed, mapping, adv = OP.expr_instance(k, 24)
    s = O.rand_fr(58, 1)[0]
    g, lag, dl, ddl = O.srs_setup(s, k)
    key = OP.keygen(c, fixed, mapping, {"g": g, "lagrange": lag, "delta": dl, "double_delta": ddl}, b"expr")
    bl = [OP.to_int(v) for v in O.rand_fr(68, OP.blind_count(c))]
    proof = OP.create_proof(key, adv, bl)
    assert OP.verify(key, proof, OP.to_int(s))
    bad = [a.copy() for a in adv]
    bad[0][3] = OP.to_mont((1 << 16) + 9)                       # a(wX) on row 2 outside the table
    with pytest.raises(ValueError):
        OP.create_proof(key, bad, bl)


@pytest.mark.parametrize("shape", ["nolookup", "bare"])
def test_circuits_without_lookup_or_permutation_verify(shape):
    """A circuit without lookups (blinding factors one fewer, no m / h / Z in
    the transcript) and one without lookups and permutation (no z either, no
    permutation polynomials in the key): the proofs verify and a witness that
    breaks a gate is rejected."""
    k = 5
    c = getattr(OP, shape + "_circuit")(k)
    fixed, mapping, adv = getattr(OP, shape + "_instance")(k, 23)
    assert OP.blinding_factors(c) == 6 and not c["lookups"]
    s = O.rand_fr(57, 1)[0]
    g, lag, dl, ddl = O.srs_setup(s, k)
    key = OP.keygen(c, fixed, mapping, {"g": g, "lagrange": lag, "delta": dl, "double_delta": ddl}, shape.encode())
    bl = [OP.to_int(v) for v in O.rand_fr(67, OP.blind_count(c))]
    proof = OP.create_proof(key, adv, bl)
    S = OP.n_perm_sets(c)
    assert S == (2 if shape == "nolookup" else 0)
    points = 4 + S + 4 + 2                                      # advice, z, limbs, f, pi
    scalars_before_q = len(c["advice_queries"]) + len(c["fixed_queries"]) + len(c["perm_cols"]) + (3 * S - 1 if S else 0)
    assert (len(proof) - 48 * points - 32 * scalars_before_q) // 32 in range(2, 8)
    assert OP.verify(key, proof, OP.to_int(s))
    bad = [a.copy() for a in adv]
    bad[2][1] = OP.to_mont(OP.to_int(bad[2][1]) + 1)           # c breaks the first gate
    assert not OP.verify(key, OP.create_proof(key, bad, bl), OP.to_int(s))


def test_generic_circuit_proofs_verify():
    """Another circuit shape: two gates as one flattened program (with a(wX)),
    four permutation columns in two sets (z of the first set opened at
    w^-(bf+1) x too), three point sets in the multi-open."""
    for k in (5, 6):
        c = OP.generic_circuit(k)
        fixed, mapping, adv = OP.generic_instance(k, k)
        s = O.rand_fr(50 + k, 1)[0]
        g, lag, dl, ddl = O.srs_setup(s, k)
        key = OP.keygen(c, fixed, mapping, {"g": g, "lagrange": lag, "delta": dl, "double_delta": ddl}, b"generic")
        assert OP.n_perm_sets(c) == 2 and key.bf == 7
        bl = [OP.to_int(v) for v in O.rand_fr(60 + k, OP.blind_count(c))]
        proof = OP.create_proof(key, adv, bl)
        assert len(proof) == 15 * 48 + 27 * 32
        assert OP.verify(key, proof, OP.to_int(s))
        bad = [a.copy() for a in adv]
        bad[2][1] = OP.to_mont(OP.to_int(bad[2][1]) + 1)          # c breaks the first gate
        assert not OP.verify(key, OP.create_proof(key, bad, bl), OP.to_int(s))
        bad = [a.copy() for a in adv]
        bad[3][1] = OP.to_mont(OP.to_int(bad[3][1]) + 1)          # d breaks the second gate
        assert not OP.verify(key, OP.create_proof(key, bad, bl), OP.to_int(s))
