"""CPU restatement of the reference's PLONK prover and verifier around the hot
path: keygen, create_proof with its Blake2b Fiat-Shamir transcript, the KZG
multi-open argument and the verifier's `prepare` with the pairing replaced by
the G1 trapdoor check.

TEST INFRASTRUCTURE ONLY: the checker for the CUDA product.  Only tests/,
__graft_entry__.smoke() and bench.py's cpu_baseline / reference legs import
this module.

Polynomials are numpy arrays of Montgomery Fr (shape (n, 4)) handled by the C
oracle (oracle.py); scalars (challenges, evaluations) are Python integers in
canonical form, so the scalar algebra of the transcript, the identities and
the verifier is independent of the C field code.  G1 points are affine
numpy arrays (12 u64, Montgomery, identity all-zero).

Circuit shape (a dict, see `config3_circuit` and `generic_circuit`): advice
and fixed columns, the reference's query lists
(`ConstraintSystem::advice_queries`/`fixed_queries`, in their order), custom
gates as a flattened program (any gates, rotations included) or the standard
gate q_l a + q_r b + q_m a b + q_o c + q_c, a permutation over advice/fixed
columns split into sets of cs.degree() - 2 columns, and at most one logup
lookup whose input is one advice column and whose table is one fixed column,
with an optional fixed selector column.  No instance columns, trashcans or
simple selectors (every identity is fully evaluated at x, so the
linearization polynomial is the quotient-limb part alone).

Randomness: the reference draws blinding values from the caller's rng in this
order: the blinding rows of every advice column (proofs/src/plonk/prover.rs:
606-617, bf + 1 each), the multiplicity blinds of every lookup (:122-123,
bf + 1 each), the permutation blinds of every set (:165-167, bf each), the
logup aggregator blinds of every lookup (:168, bf each).  The quotient-limb
blinds come from OsRng in the reference (prover.rs:774-785); here they are the
next qdeg - 1 values of the same stream, a documented deviation that makes
proofs reproducible.
"""
import hashlib

import numpy as np

from . import oracle as O

R = 0x73EDA753299D7D483339D80809A1D80553BDA402FFFE5BFEFFFFFFFF00000001
P_BASE = 0x1A0111EA397FE69A4B1BA7B6434BACD764774B84F38512BF6730D2A0F6B0F6241EABFFFEB153FFFFB9FEFFFFFFFFAAAB
MONT = pow(2, 256, R)
MONT_INV = pow(MONT, -1, R)
TRANSCRIPT_KEY = b"Domain separator for transcript"   # transcript/implementors.rs:18
VK_PERSONAL = b"Halo2-Verify-Key"                     # plonk/mod.rs:244-245
VK_VERSION = 0x03                                     # plonk/mod.rs:74


# ------------------------------------------------------------ field helpers --
def to_int(a):
    """Montgomery Fr (4 u64) -> canonical integer."""
    a = np.asarray(a, np.uint64)
    v = int(a[0]) | int(a[1]) << 64 | int(a[2]) << 128 | int(a[3]) << 192
    return v * MONT_INV % R


def to_mont(v):
    """canonical integer -> Montgomery Fr (4 u64)."""
    m = (v % R) * MONT % R
    return np.array([(m >> (64 * i)) & 0xFFFFFFFFFFFFFFFF for i in range(4)], np.uint64)


def from_uniform_bytes(b64):
    """Fq::from_uniform_bytes (curves/src/bls12_381/fq.rs:712-736): a0*R^2 +
    a1*R^3 in Montgomery form, i.e. the 512-bit little-endian integer mod r."""
    return int.from_bytes(b64, "little") % R


def inv(v):
    return pow(v, R - 2, R)


def powers(base, count):
    """utils/arithmetic.rs:266-268."""
    out, p = [], 1
    for _ in range(count):
        out.append(p)
        p = p * base % R
    return out


# ------------------------------------------------------------ G1 encodings --
def _fp_canon_int(limbs6):
    return O.to_int(O.fp_op("to_canonical", np.asarray(limbs6, np.uint64)))


def is_identity(aff):
    return not np.any(np.asarray(aff, np.uint64))


def compress(aff):
    """GroupEncoding::to_bytes of G1 (ZCash compressed, g1.rs:326-334)."""
    return bytes(O.g1_compress(np.asarray(aff, np.uint64)))


def uncompressed(aff):
    """G1Affine::to_uncompressed (SerdeFormat::RawBytesUnchecked writes of the
    VK hash, plonk/mod.rs:252-262; g1.rs:486-488): x, y big-endian, 0x40 flag
    for the identity."""
    if is_identity(aff):
        return bytes([0x40]) + bytes(95)
    x, y = _fp_canon_int(aff[:6]), _fp_canon_int(aff[6:])
    return x.to_bytes(48, "big") + y.to_bytes(48, "big")


def pt_mul(aff, s):
    if is_identity(aff) or s % R == 0:
        return np.zeros(12, np.uint64)
    return O.g1_mul(np.asarray(aff, np.uint64), to_mont(s))


def pt_add(a, b):
    return O.g1_to_affine(O.g1_jac_add(O.g1_from_affine(a), O.g1_from_affine(b)))


def pt_lincomb(points, scalars):
    acc = np.zeros(12, np.uint64)
    for p, s in zip(points, scalars):
        acc = pt_add(acc, pt_mul(p, s))
    return acc


# ------------------------------------------------------------- transcript --
class Transcript:
    """CircuitTranscript<Blake2bState> (transcript/mod.rs:83-150,
    implementors.rs:13-30): one keyed Blake2b-512 state; absorbing prefixes a
    1 byte, squeezing absorbs a 0 byte and reads the digest without resetting
    the state; G1 points go in compressed (48 bytes), scalars as 32-byte
    little-endian canonical values (implementors.rs:138-175); a challenge is
    the 64-byte digest reduced mod r (implementors.rs:177-185)."""

    def __init__(self, proof=b""):
        self.h = hashlib.blake2b(digest_size=64, key=TRANSCRIPT_KEY)
        self.proof = bytearray()
        self.buf, self.pos = bytes(proof), 0

    def common_bytes(self, b):
        self.h.update(b"\x01" + b)

    def common_fr(self, v):
        self.common_bytes((v % R).to_bytes(32, "little"))

    def write_fr(self, v):
        b = (v % R).to_bytes(32, "little")
        self.common_bytes(b)
        self.proof += b

    def write_point(self, aff):
        b = compress(aff)
        self.common_bytes(b)
        self.proof += b

    def squeeze(self):
        self.h.update(b"\x00")
        return from_uniform_bytes(self.h.digest())

    # verifier side (Transcript::read, mod.rs:128-133)
    def read_fr(self):
        b = self.buf[self.pos:self.pos + 32]
        if len(b) != 32:
            raise ValueError("proof too short")
        v = int.from_bytes(b, "little")
        if v >= R:
            raise ValueError("non-canonical scalar")
        self.pos += 32
        self.common_bytes(b)
        return v

    def read_point(self):
        b = self.buf[self.pos:self.pos + 48]
        if len(b) != 48:
            raise ValueError("proof too short")
        st, aff = O.g1_decompress(b, True)
        if st != 0:
            raise ValueError(f"invalid point encoding ({st})")
        self.pos += 48
        self.common_bytes(b)
        return aff

    def assert_empty(self):
        if self.pos != len(self.buf):
            raise ValueError("trailing bytes")


# ---------------------------------------------------------------- circuit --
def blinding_factors(circuit):
    """ConstraintSystem::blinding_factors (plonk/circuit.rs:2203-2245) for this
    shape: max(3, max advice queries per column) + trashcans + helper chunks
    + 3."""
    per_col = {}
    for col, _ in circuit["advice_queries"]:
        per_col[col] = per_col.get(col, 0) + 1
    f = max(3, max(per_col.values(), default=1))
    return f + len(circuit.get("trashcans", [])) + sum(len(lookup_chunks(circuit, lk)) for lk in circuit["lookups"]) + 3


def n_perm_sets(circuit):
    chunk = circuit["degree"] - 2
    return (len(circuit["perm_cols"]) + chunk - 1) // chunk


def blind_count(circuit):
    """Number of rng values one proof draws (the order in the module doc)."""
    bf = blinding_factors(circuit)
    qdeg = circuit["degree"] - 1
    L = len(circuit["lookups"])
    return circuit["n_advice"] * (bf + 1) + L * (bf + 1) + n_perm_sets(circuit) * bf + L * bf + (qdeg - 1)


def query_index(queries, col, rot=0):
    """ConstraintSystem::get_any_query_index for the column at rotation rot."""
    for i, (c, r) in enumerate(queries):
        if c == col and r == rot:
            return i
    raise KeyError((col, rot))


def config3_circuit(k):
    """The single-proof configuration: advice a, b, c, fixed q_l, q_r, q_m,
    q_o, q_c, the lookup table and the lookup selector; the standard gate;
    the permutation over a, b, c; one lookup of a into the table; degree 5
    (set_minimum_degree(5), proofs/benches/plonk.rs:191)."""
    return {
        "k": k, "degree": 5, "n_advice": 3, "n_fixed": 7,
        "advice_queries": [(0, 0), (1, 0), (2, 0)],
        "fixed_queries": [(i, 0) for i in range(7)],
        "gate_fixed": [0, 1, 2, 3, 4], "gate_advice": [0, 1, 2],
        "perm_cols": [(0, 0), (0, 1), (0, 2)],          # (0 advice | 1 fixed, column)
        "lookups": [{"input": 0, "table": 5, "selector": 6}],
    }


def config3_instance(k, seed, table_bits=16, copy_fraction=0.10):
    """Seeded fixed columns, copy cycles and a satisfying witness for
    config3_circuit: selectors uniform (q_o non-zero) on the usable rows and
    zero on the rest; the table holds 0 .. 2^table_bits - 1 (capped at the
    usable rows) padded with zeros; a is a table value, b uniform, c solves the
    gate; copy cycles over copy_fraction of the a and b cells of usable rows,
    each cycle carrying one table value.  Returns (fixed_values, mapping,
    advice_values) with mapping[c][r] = (column, row) of the next cell of
    (c, r)'s cycle (identity elsewhere), the permutation build_pk takes
    (permutation/keygen.rs:138-185)."""
    c = config3_circuit(k)
    n = 1 << k
    bf = blinding_factors(c)
    u = n - bf - 1
    rng = np.random.default_rng(seed)
    rows = min(1 << table_bits, u)
    col = lambda s: O.rand_fr(seed * 97 + s, n)
    q = [col(i) for i in range(5)]
    for qi in q:
        qi[u:] = 0
    one = O.fr_const(0)
    # q_o non-zero on usable rows (a zero draw has negligible probability; replace it anyway)
    for i in range(u):
        if not np.any(q[3][i]):
            q[3][i] = one
    table = np.zeros((n, 4), np.uint64)
    table[:rows] = np.stack([to_mont(v) for v in range(rows)]) if rows else table[:0]
    sel = np.zeros((n, 4), np.uint64)
    sel[:u] = one
    fixed = q + [table, sel]
    a_int = rng.integers(0, rows, size=u)
    a = np.zeros((n, 4), np.uint64)
    b = col(10)
    b[u:] = 0
    # copy cycles among the a and b cells of usable rows
    mapping = np.zeros((3, n, 2), np.uint32)
    for ci in range(3):
        mapping[ci, :, 0] = ci
        mapping[ci, :, 1] = np.arange(n, dtype=np.uint32)
    cells = rng.permutation(2 * u)[: int(copy_fraction * 2 * u)]
    pos = 0
    cyc_vals = {}
    while pos + 1 < len(cells):
        ln = int(rng.integers(2, 5))
        cyc = cells[pos:pos + ln]
        pos += ln
        if len(cyc) < 2:
            break
        v = int(rng.integers(0, rows))
        for t, cell in enumerate(cyc):
            nxt = cyc[(t + 1) % len(cyc)]
            cc, rr = divmod(int(cell), u)
            mapping[cc, rr] = divmod(int(nxt), u)
            cyc_vals[(cc, rr)] = v
    for (cc, rr), v in cyc_vals.items():
        if cc == 0:
            a_int[rr] = v
        else:
            b[rr] = to_mont(v)
    a[:u] = np.stack([to_mont(int(v)) for v in a_int])
    # c = -(q_l a + q_r b + q_m a b + q_c) / q_o on usable rows
    t = O.poly_inner_product([_hadamard(q[0], a), _hadamard(q[1], b), _hadamard(q[2], _hadamard(a, b)), q[4]],
                             [one] * 4)
    cc_col = _hadamard(O.poly_inner_product([t], [to_mont(R - 1)]), O.batch_invert(q[3]))
    cc_col[u:] = 0
    return fixed, mapping, [a, b, cc_col]


def generic_circuit(k, two_lookups=False):
    """A circuit of another shape: advice a, b, c, d with a queried at rotations
    0 and 1, fixed q1, q2, q3, q4, the table and the lookup selector; two gates
    as one flattened program, q1 a b + q2 a(wX) - q4 c and q3 (d - a^2), folded
    by Horner in y; the permutation over a, b, c, d (two sets of three and one
    columns); a lookup of a into the table; degree 5.  two_lookups: a seventh
    fixed column, the table of squares, and a second lookup, of d into it
    without a selector."""
    zero, one = to_mont(0), to_mont(1)
    gates = {"constants": [zero, one], "rotations": [0, 1],
             # values: constants 0, 1; slots beta 2, theta 3, trash 4, y 5, previous 6; reads 7..15
             "reads": [(0, 0, 0, 7), (0, 1, 0, 8), (0, 2, 0, 9), (0, 3, 0, 10), (1, 0, 0, 11), (1, 1, 0, 12),
                       (1, 2, 0, 13), (1, 3, 0, 14), (1, 0, 1, 15)],
             "ops": [(2, 16, 11, 12, 0), (2, 17, 7, 16, 0), (2, 18, 8, 15, 0), (0, 19, 17, 18, 0),
                     (2, 20, 10, 13, 0), (1, 21, 19, 20, 0), (3, 22, 11, 0, 0), (1, 23, 14, 22, 0),
                     (2, 24, 9, 23, 0), (6, 25, 6, 5, 21), (6, 26, 25, 5, 24)],
             "values_len": 27, "beta_idx": 2, "theta_idx": 3, "trash_challenge_idx": 4, "y_idx": 5,
             "previous_value_idx": 6, "result_idx": 26}
    nf = 7 if two_lookups else 6
    lookups = [{"input": 0, "table": 4, "selector": 5}]
    if two_lookups:
        lookups.append({"input": 3, "table": 6, "selector": None})
    return {"k": k, "degree": 5, "n_advice": 4, "n_fixed": nf,
            "advice_queries": [(0, 0), (1, 0), (2, 0), (3, 0), (0, 1)],
            "fixed_queries": [(i, 0) for i in range(nf)],
            "gates": gates,
            "perm_cols": [(0, 0), (0, 1), (0, 2), (0, 3)],
            "lookups": lookups}


def _cycles(rng, n, u, n_cols, cycle_cols, fraction, rows):
    """Copy cycles of 2 to 4 cells over `fraction` of the cells of columns
    cycle_cols in rows [0, u): (mapping (n_cols, n, 2), {(col, row): value})
    with one table value in [0, rows) per cycle."""
    mapping = np.zeros((n_cols, n, 2), np.uint32)
    for ci in range(n_cols):
        mapping[ci, :, 0] = ci
        mapping[ci, :, 1] = np.arange(n, dtype=np.uint32)
    ncyc = len(cycle_cols)
    cells = rng.permutation(ncyc * u)[: int(fraction * ncyc * u)]
    pos, vals = 0, {}
    while pos + 1 < len(cells):
        ln = int(rng.integers(2, 5))
        cyc = cells[pos:pos + ln]
        pos += ln
        if len(cyc) < 2:
            break
        v = int(rng.integers(0, rows))
        for t, cell in enumerate(cyc):
            nxt = cyc[(t + 1) % len(cyc)]
            cc, rr = divmod(int(cell), u)
            nc, nr = divmod(int(nxt), u)
            mapping[cycle_cols[cc], rr] = (cycle_cols[nc], nr)
            vals[(cycle_cols[cc], rr)] = v
    return mapping, vals


def generic_instance(k, seed, table_bits=16, copy_fraction=0.10, two_lookups=False, circuit=None):
    """Seeded fixed columns, copy cycles (over the a and b cells of rows
    before the last usable row) and a satisfying witness of generic_circuit:
    a a table value, b uniform, c = q1 a b + q2 a(wX), d = a^2; the gate
    selectors q1, q2, q4 are zero from the last usable row on (its a(wX) is a
    blinding row), q3 from the usable rows on.  two_lookups: the table of
    squares t2[i] = i^2 (i < the table's rows; zero after), which holds every
    usable d.  circuit: the circuit whose blinding factors fix the usable rows
    (default generic_circuit's)."""
    c = circuit if circuit is not None else generic_circuit(k, two_lookups)
    n = 1 << k
    bf = blinding_factors(c)
    u = n - bf - 1
    rng = np.random.default_rng(seed)
    rows = min(1 << table_bits, u)
    one = O.fr_const(0)
    q = [O.rand_fr(seed * 131 + i, n) for i in range(3)]
    q1, q2, q3 = q
    q1[u - 1:] = 0
    q2[u - 1:] = 0
    q3[u:] = 0
    q4 = np.zeros((n, 4), np.uint64)
    q4[:u - 1] = one
    table = np.zeros((n, 4), np.uint64)
    table[:rows] = np.stack([to_mont(v) for v in range(rows)])
    sel = np.zeros((n, 4), np.uint64)
    sel[:u] = one
    mapping, vals = _cycles(rng, n, u - 1, 4, [0, 1], copy_fraction, rows)
    a_int = rng.integers(0, rows, size=u)
    b = O.rand_fr(seed * 131 + 7, n)
    b[u:] = 0
    for (cc, rr), v in vals.items():
        if cc == 0:
            a_int[rr] = v
        else:
            b[rr] = to_mont(v)
    a = np.zeros((n, 4), np.uint64)
    a[:u] = np.stack([to_mont(int(v)) for v in a_int])
    a_next = np.zeros_like(a)
    a_next[:-1] = a[1:]
    cc_col = O.poly_inner_product([_hadamard(q1, _hadamard(a, b)), _hadamard(q2, a_next)], [one, one])
    cc_col[u - 1:] = 0
    d = _hadamard(a, a)
    d[u:] = 0
    fixed = [q1, q2, q3, q4, table, sel]
    if two_lookups:
        squares = np.zeros((n, 4), np.uint64)
        squares[:rows] = np.stack([to_mont(v * v) for v in range(rows)])
        fixed.append(squares)
    return fixed, mapping, [a, b, cc_col, d]


def instance_circuit(k):
    """generic_circuit with one instance column (public inputs): a third gate
    q5 (c - inst) over a seventh fixed column q5, and the instance column as a
    fifth permutation column whose first rows are copies of c's."""
    c = generic_circuit(k)
    g = dict(c["gates"])
    g["reads"] = g["reads"] + [(0, 6, 0, 27), (2, 0, 0, 28)]
    g["ops"] = g["ops"] + [(1, 29, 13, 28, 0), (2, 30, 27, 29, 0), (6, 31, 26, 5, 30)]
    g["values_len"], g["result_idx"] = 32, 31
    c.update({"gates": g, "n_fixed": 7, "fixed_queries": [(i, 0) for i in range(7)], "n_instance": 1,
              "instance_queries": [(0, 0)], "perm_cols": c["perm_cols"] + [(2, 0)]})
    return c


def tuple_circuit(k):
    """generic_circuit whose lookup takes the tuple (a, d) into the tuple
    (table, table of squares), both compressed with theta, with the selector
    column: the multi-column table lookup."""
    c = generic_circuit(k, two_lookups=True)
    c["lookups"] = [{"input": [0, 3], "table": [4, 6], "selector": 5}]
    return c


def tuple_instance(k, seed):
    return generic_instance(k, seed, two_lookups=True, circuit=tuple_circuit(k))


def nolookup_circuit(k):
    """generic_circuit without its lookup: no multiplicity, helper or
    aggregator commitments, and one blinding factor fewer."""
    c = generic_circuit(k)
    c["lookups"] = []
    return c


def nolookup_instance(k, seed):
    return generic_instance(k, seed, circuit=nolookup_circuit(k))


def bare_circuit(k):
    """generic_circuit with neither its lookup nor its permutation: the
    gates alone (no z, m, h or Z commitments, no permutation polynomials in
    the key)."""
    c = nolookup_circuit(k)
    c["perm_cols"] = []
    return c


def bare_instance(k, seed):
    fixed, mapping, adv = generic_instance(k, seed, circuit=bare_circuit(k))
    return fixed, mapping[:0], adv


def _expr_program(rotations, reads, ops, values_len, result_idx):
    """A lookup input expression as a flattened program: constants 0 and 1,
    challenge slots 2-6 (beta, theta, trash challenge, y, previous value)."""
    return {"constants": [to_mont(0), to_mont(1)], "rotations": rotations, "reads": reads, "ops": ops,
            "values_len": values_len, "beta_idx": 2, "theta_idx": 3, "trash_challenge_idx": 4, "y_idx": 5,
            "previous_value_idx": 6, "result_idx": result_idx}


def expr_circuit(k):
    """generic_circuit with the table of squares and lookups whose inputs are
    expressions: a(wX) and d - a^2 + a into the table, selected by q4 (one on
    the rows before the last usable one, where a(wX) is still a table value;
    the second input has degree 2, so a helper takes two inputs at degree 5),
    and the tuple (a, a * a) into (table, squares) without a selector."""
    c = generic_circuit(k, two_lookups=True)
    a_next = _expr_program([0, 1], [(1, 0, 1, 7)], [], 8, 7)
    d_minus = _expr_program([0], [(1, 3, 0, 7), (1, 0, 0, 8)], [(2, 9, 8, 8, 0), (1, 10, 7, 9, 0), (0, 11, 10, 8, 0)],
                            12, 11)
    a_sq = _expr_program([0], [(1, 0, 0, 7)], [(3, 8, 7, 0, 0)], 9, 8)
    c["lookups"] = [{"inputs": [[a_next], [d_minus]], "table": 4, "selector": 3},
                    {"input": [0, a_sq], "table": [4, 6], "selector": None}]
    return c


def expr_instance(k, seed):
    return generic_instance(k, seed, two_lookups=True, circuit=expr_circuit(k))


def parallel_circuit(k):
    """generic_circuit with the table of squares and three more advice
    columns e, f, g (queried at rotation 0, in no gate nor permutation), and
    two lookups with parallel inputs: a, e, f, a, e into the table with the
    selector (five inputs: two helper chunks at degree 5, of four and one),
    and the tuples (a, d), (e, g) into (table, squares) without a selector
    (one chunk of two theta-compressed inputs)."""
    c = generic_circuit(k, two_lookups=True)
    c["n_advice"] = 7
    c["advice_queries"] = c["advice_queries"] + [(4, 0), (5, 0), (6, 0)]
    c["lookups"] = [{"inputs": [0, 4, 5, 0, 4], "table": 4, "selector": 5},
                    {"inputs": [[0, 3], [4, 6]], "table": [4, 6], "selector": None}]
    return c


def parallel_instance(k, seed):
    """generic_instance's columns with e, f table values on the usable rows
    and g = e^2 (zero past the usable rows)."""
    c = parallel_circuit(k)
    fixed, mapping, adv = generic_instance(k, seed, two_lookups=True, circuit=c)
    n = 1 << k
    u = n - blinding_factors(c) - 1
    rows = min(1 << 16, u)
    rng = np.random.default_rng(seed + 77)
    e, f = (np.zeros((n, 4), np.uint64) for _ in range(2))
    e[:u] = np.stack([to_mont(int(v)) for v in rng.integers(0, rows, size=u)])
    f[:u] = np.stack([to_mont(int(v)) for v in rng.integers(0, rows, size=u)])
    g = _hadamard(e, e)
    g[u:] = 0
    return fixed, mapping, adv + [e, f, g]


def selector_circuit(k):
    """generic_circuit with q3 a simple selector: its second gate
    polynomial q3 (d - a^2) is listed with q3 as selector, so q3 is evaluated
    as one at x, not written to the transcript nor opened, and its fixed
    polynomial enters the linearization scaled by d(x) - a(x)^2."""
    c = generic_circuit(k)
    c["gate_polys"] = [(21, None), (24, 2)]
    return c


def selector_instance(k, seed):
    """generic_instance with the simple selector q3 boolean: one on the usable
    rows."""
    fixed, mapping, adv = generic_instance(k, seed, circuit=selector_circuit(k))
    n = 1 << k
    u = n - blinding_factors(selector_circuit(k)) - 1
    q3 = np.zeros((n, 4), np.uint64)
    q3[:u] = O.fr_const(0)
    fixed = list(fixed)
    fixed[2] = q3
    return fixed, mapping, adv


def trash_circuit(k):
    """generic_circuit with a trashcan (trash.rs): constraint expressions
    d - a^2 and q1 a b + q2 a(wX) - q4 c folded with the trash challenge, the
    selector q3 (non-zero only on rows where both vanish).  With the
    trashcan the lookup goes to the quotient as a helper program."""
    zero, one = to_mont(0), to_mont(1)
    program = {"constants": [zero, one], "rotations": [0, 1],
               # values: constants 0, 1; slots beta 2, theta 3, trash 4, y 5, previous 6; reads 7..14
               "reads": [(0, 0, 0, 7), (0, 1, 0, 8), (0, 3, 0, 9), (1, 0, 0, 10), (1, 1, 0, 11), (1, 2, 0, 12),
                         (1, 3, 0, 13), (1, 0, 1, 14)],
               "ops": [(2, 15, 10, 11, 0), (2, 16, 7, 15, 0), (2, 17, 8, 14, 0), (0, 18, 16, 17, 0),
                       (2, 19, 9, 12, 0), (1, 20, 18, 19, 0), (3, 21, 10, 0, 0), (1, 22, 13, 21, 0),
                       (6, 23, 6, 4, 22), (6, 24, 23, 4, 20)],
               "values_len": 25, "beta_idx": 2, "theta_idx": 3, "trash_challenge_idx": 4, "y_idx": 5,
               "previous_value_idx": 6, "result_idx": 24}
    c = generic_circuit(k)
    c["trashcans"] = [{"program": program, "selector": 2}]
    return c


def trash_instance(k, seed):
    return generic_instance(k, seed, circuit=trash_circuit(k))


def many_circuit(k):
    """generic_circuit with the table of squares, five lookups (a into the
    table with and without the selector, d into the squares with and
    without it, the tuple (a, d) into (table, squares) with q4) and five
    trashcans (trash_circuit's program, each with its own selector column
    among q3 and the lookup selector): more lookups and trashcans than a
    smaller key takes."""
    c = generic_circuit(k, two_lookups=True)
    c["lookups"] = [{"input": 0, "table": 4, "selector": 5}, {"input": 3, "table": 6, "selector": None},
                    {"input": 0, "table": 4, "selector": None}, {"input": 3, "table": 6, "selector": 5},
                    {"input": [0, 3], "table": [4, 6], "selector": 3}]
    program = trash_circuit(k)["trashcans"][0]["program"]
    c["trashcans"] = [{"program": program, "selector": sel} for sel in (2, 2, 5, 2, 5)]
    return c


def many_instance(k, seed):
    return generic_instance(k, seed, two_lookups=True, circuit=many_circuit(k))


INSTANCE_ROWS = 3


def instance_instance(k, seed):
    """generic_instance's columns and witness with q5 = 1 on the first
    INSTANCE_ROWS rows, the public values inst_i = c_i there, and copy
    constraints between each instance cell and its c cell.  Returns
    (fixed, mapping, advice, instances)."""
    fixed, mapping, adv = generic_instance(k, seed)
    n = 1 << k
    q5 = np.zeros((n, 4), np.uint64)
    q5[:INSTANCE_ROWS] = O.fr_const(0)
    fixed = fixed + [q5]
    m = np.zeros((5, n, 2), np.uint32)
    m[:4] = mapping
    m[4, :, 0] = 4
    m[4, :, 1] = np.arange(n, dtype=np.uint32)
    for r in range(INSTANCE_ROWS):
        m[4, r] = (2, r)
        m[2, r] = (4, r)
    inst = [adv[2][:INSTANCE_ROWS].copy()]
    return fixed, m, adv, inst


def generic2_circuit(k):
    """generic_circuit with its second lookup (d into the table of squares)."""
    return generic_circuit(k, two_lookups=True)


def generic2_instance(k, seed):
    return generic_instance(k, seed, two_lookups=True)


def _hadamard(x, y):
    """Element-wise product of two Fr arrays (through the C oracle)."""
    return O.fr_mul_vec(x, y)


# ------------------------------------------------------------- polynomials --
def delta(a, order):
    """Polynomial::to_delta / to_double_delta (proofs/src/poly/mod.rs:297-336)."""
    a = np.ascontiguousarray(a, np.uint64)
    one, m1 = O.fr_const(0), to_mont(R - 1)
    out = a.copy()
    shifted = np.zeros_like(a)
    shifted[1:] = a[:-1]
    out = O.poly_inner_product([a, shifted], [one, m1])
    if order == 2:
        s2 = np.zeros_like(out)
        s2[1:] = out[:-1]
        out = O.poly_inner_product([out, s2], [one, m1])
    return out


def commit(scalars, bases):
    """KZGCommitmentScheme::commit_many's msm_specific over bases[..len]
    (kzg/mod.rs:82-108)."""
    scalars = np.ascontiguousarray(scalars, np.uint64)
    return O.msm_specific(scalars, np.ascontiguousarray(bases[: scalars.shape[0]], np.uint64))


def scale(poly, s):
    return O.poly_inner_product([poly], [to_mont(s)])


def eval_at(poly, point):
    return to_int(O.eval_polynomial(poly, to_mont(point)))


def compute_multiplicities(selector, inputs, table, usable_rows, blinds):
    """logup/prover.rs:412-477: per table row, the number of selected input
    rows holding its value divided by the value's count in the table (active
    rows only); blinding rows take the blinding values.  Raises when a
    selected input value is not in the table."""
    n = table.shape[0]
    vt = np.dtype((np.void, 32))
    tab = np.ascontiguousarray(table[:usable_rows]).view(vt).ravel()
    uniq, inv_idx, counts = np.unique(tab, return_inverse=True, return_counts=True)
    incount = np.zeros(len(uniq), np.int64)
    sel = np.any(selector[:usable_rows] != 0, axis=1)
    for col in inputs:
        iv = np.ascontiguousarray(col[:usable_rows][sel]).view(vt).ravel()
        pos = np.searchsorted(uniq, iv)
        ok = (pos < len(uniq))
        ok[ok] = uniq[pos[ok]] == iv[ok]
        if not np.all(ok):
            raise ValueError("input value not found in lookup table")
        incount += np.bincount(pos, minlength=len(uniq))
    vals = np.stack([to_mont(int(incount[i]) * inv(int(counts[i])) % R) for i in range(len(uniq))])
    m = np.zeros((n, 4), np.uint64)
    m[:usable_rows] = vals[inv_idx.ravel()]
    m[usable_rows:] = np.stack([to_mont(v) for v in blinds])
    return m


# ------------------------------------------------------------------ keygen --
class Key:
    pass


def keygen(circuit, fixed_values, mapping, srs, pinned_repr):
    """keygen_vk / keygen_pk for this shape (plonk/keygen.rs:227-359):
    fixed polynomials and cosets, the permutation polynomials of build_pk
    (permutation/keygen.rs:138-185: cell (c, r) gets delta^c' omega^r' of the
    cell it maps to), their polynomials and cosets, l0, l_last and
    l_active_row (keygen.rs:361-404), the fixed and permutation commitments
    and the VK's transcript_repr (plonk/mod.rs:227-284).  srs: dict with the
    affine bases g, lagrange, delta, double_delta (n points each).
    pinned_repr: the bytes of format!("{:?}", domain.pinned()) followed by
    format!("{:?}", cs.pinned()), which this restatement cannot produce (they
    are Rust Debug strings) and takes as given."""
    key = Key()
    k = circuit["k"]
    n = 1 << k
    dom = O.Domain(circuit["degree"], k)
    bf = blinding_factors(circuit)
    key.circuit, key.dom, key.srs, key.n, key.bf = circuit, dom, srs, n, bf
    key.u = n - bf - 1
    key.qdeg = circuit["degree"] - 1
    key.omega, key.omega_inv = to_int(dom.get(0)), to_int(dom.get(1))
    key.fixed_values = [np.ascontiguousarray(v, np.uint64) for v in fixed_values]
    key.fixed_polys = [dom.lagrange_to_coeff(v) for v in key.fixed_values]
    key.fixed_cosets = [dom.coeff_to_extended(p) for p in key.fixed_polys]
    # permutation polynomials: deltaomega[c][r] = delta^c * omega^r
    x_poly = np.zeros((n, 4), np.uint64)
    x_poly[1] = O.fr_const(0)
    omega_pows = dom.coeff_to_lagrange(x_poly)          # omega^r, r = 0..n-1
    P = len(circuit["perm_cols"])
    dlt = to_int(O.fr_const(5))
    deltaomega = np.stack([scale(omega_pows, pow(dlt, c, R)) for c in range(P)]) if P else None
    if mapping is None:
        mapping = np.zeros((P, n, 2), np.uint32)
        for c in range(P):
            mapping[c, :, 0] = c
            mapping[c, :, 1] = np.arange(n)
    key.perm_values = [np.ascontiguousarray(deltaomega[mapping[c, :, 0], mapping[c, :, 1]]) for c in range(P)]
    key.perm_polys = [dom.lagrange_to_coeff(v) for v in key.perm_values]
    key.perm_cosets = [dom.coeff_to_extended(p) for p in key.perm_polys]
    # l0, l_last, l_active_row
    one = O.fr_const(0)
    unit = lambda rows: _unit(n, rows)
    l0 = dom.coeff_to_extended(dom.lagrange_to_coeff(unit([0])))
    l_blind = dom.coeff_to_extended(dom.lagrange_to_coeff(unit(range(n - bf, n))))
    l_last = dom.coeff_to_extended(dom.lagrange_to_coeff(unit([n - bf - 1])))
    ones = np.tile(one, (l0.shape[0], 1))
    l_active = O.poly_inner_product([ones, l_last, l_blind], [one, to_mont(R - 1), to_mont(R - 1)])
    key.l0, key.l_last, key.l_active = l0, l_last, l_active
    # commitments and the VK hash
    key.fixed_coms = [commit(v, srs["lagrange"]) for v in key.fixed_values]
    key.perm_coms = [commit(v, srs["lagrange"]) for v in key.perm_values]
    key.repr = vk_transcript_repr(k, key.fixed_coms, key.perm_coms, pinned_repr)
    # lookup table index of the multiplicities
    return key


def _unit(n, rows):
    a = np.zeros((n, 4), np.uint64)
    for r in rows:
        a[r] = O.fr_const(0)
    return a


def vk_transcript_repr(k, fixed_coms, perm_coms, pinned_repr):
    """VerifyingKey::from_parts (plonk/mod.rs:227-284): Blake2b-512 with the
    personalisation "Halo2-Verify-Key" over the version byte, k, the fixed
    and permutation commitments (uncompressed, each list prefixed by its u32
    length) and the pinned Debug strings, then from_uniform_bytes."""
    buf = bytearray([VK_VERSION, k]) + len(fixed_coms).to_bytes(4, "little")
    for c in fixed_coms:
        buf += uncompressed(c)
    buf += len(perm_coms).to_bytes(4, "little")
    for c in perm_coms:
        buf += uncompressed(c)
    buf += pinned_repr
    return from_uniform_bytes(hashlib.blake2b(bytes(buf), digest_size=64, person=VK_PERSONAL).digest())


def vk_bytes(key, processed=True):
    """VerifyingKey::write (plonk/mod.rs:95-113): version, k, the u32 LE count
    and the fixed commitments, then the permutation commitments; points
    compressed (SerdeFormat::Processed) or uncompressed (RawBytes*)
    (utils/helpers.rs:94-104)."""
    enc = compress if processed else uncompressed
    out = bytearray([VK_VERSION, key.circuit["k"]]) + len(key.fixed_coms).to_bytes(4, "little")
    for c in key.fixed_coms + key.perm_coms:
        out += enc(c)
    return bytes(out)


def pk_bytes(key, processed=True):
    """ProvingKey::write (plonk/mod.rs:391-399): the VK, then the fixed
    columns' values and the permutation polynomials' values as polynomial
    slices (u32 BE count, per polynomial a u32 BE length and the raw Montgomery
    limbs, helpers.rs:150-160, poly/mod.rs:544-550, fq.rs:912-917)."""
    out = bytearray(vk_bytes(key, processed))
    for cols in (key.fixed_values, key.perm_values):
        out += len(cols).to_bytes(4, "big")
        for c in cols:
            out += c.shape[0].to_bytes(4, "big") + np.ascontiguousarray(c, "<u8").tobytes()
    return bytes(out)


# ------------------------------------------------------- shared identities --
def l_i_range(key, x, xn, rotations):
    """EvaluationDomain::l_i_range (domain.rs:487-512): l_i(x) =
    omega^i (x^n - 1) / (n (x - omega^i))."""
    n = key.n
    out = []
    for rot in rotations:
        wi = pow(key.omega, rot, R) if rot >= 0 else pow(key.omega_inv, -rot, R)
        out.append(wi * (xn - 1) % R * inv(n) % R * inv((x - wi) % R) % R)
    return out


def instance_evals(key, instances, x, xn):
    """The instance query evaluations of the verifier (verifier.rs:205-242):
    for the query (column, rotation), sum_j value_j l_{j - rotation}(x),
    the Lagrange basis of the rows the values occupy."""
    out = []
    for col, rot in key.circuit.get("instance_queries", []):
        vals = [to_int(v) for v in np.ascontiguousarray(instances[col], np.uint64).reshape(-1, 4)]
        ls = l_i_range(key, x, xn, range(-rot, len(vals) - rot))
        out.append(sum(v * li for v, li in zip(vals, ls)) % R)
    return out


def rotate(key, x, rot):
    """EvaluationDomain::rotate_omega (domain.rs:449-457)."""
    return x * (pow(key.omega, rot, R) if rot >= 0 else pow(key.omega_inv, -rot, R)) % R


def identities(key, ev, ch):
    """partially_evaluate_identities (plonk/mod.rs:519-608) with every
    identity fully evaluated: the gate polynomials, then the permutation
    expressions (permutation.rs:195-290), then each lookup's boundary, helper
    and accumulator expressions (logup.rs:405-485).  ev: evaluations by name;
    ch: challenges.  Returns the identities in order, each with the fixed
    column of its simple selector (None: fully evaluated); a simple
    selector's evaluation in ev["fixed"] is one (verifier.rs:250-259)."""
    c = key.circuit
    x, xn, beta, gamma, theta = ch["x"], ch["xn"], ch["beta"], ch["gamma"], ch["theta"]
    bf = key.bf
    l_evals = l_i_range(key, x, xn, range(-(bf + 1), 1))
    l_last, l_blind, l_0 = l_evals[0], sum(l_evals[1:1 + bf]) % R, l_evals[1 + bf]
    adv, fix, ins = ev["advice"], ev["fixed"], ev.get("instance", [])
    aq = lambda col: adv[query_index(c["advice_queries"], col)]
    fq = lambda col: fix[query_index(c["fixed_queries"], col)]
    iq = lambda col: ins[query_index(c.get("instance_queries", []), col)]
    col_eval = lambda kind, col: (aq, fq, iq)[kind](col)

    def read_query(col_type, col, rot):
        qs = (c["fixed_queries"], c["advice_queries"], c.get("instance_queries", []))[col_type]
        return (fix, adv, ins)[col_type][query_index(qs, col, rot)]
    # a lookup input element at x: its advice column's evaluation, or its expression's value
    lookup_input_at = lambda el: aq(el) if is_column(el) else program_at(el, read_query, ch)
    if c.get("gates") is not None:
        def read(col_type, col, rot):
            if col_type == 0:
                return fix[query_index(c["fixed_queries"], col, rot)]
            if col_type == 2:
                return ins[query_index(c.get("instance_queries", []), col, rot)]
            return adv[query_index(c["advice_queries"], col, rot)]
        if c.get("gate_polys"):
            vals = program_at(c["gates"], read, ch, all_values=True)
            out = [(sel, vals[slot]) for slot, sel in c["gate_polys"]]
        else:
            out = [(None, program_at(c["gates"], read, ch))]
    else:
        gf, ga = c["gate_fixed"], c["gate_advice"]
        ql, qr, qm, qo, qc = (fq(i) for i in gf)
        a, b, cc = (aq(i) for i in ga)
        out = [(None, (ql * a + qr * b + qm * a * b + qo * cc + qc) % R)]
    # permutation
    sets = ev["perm_sets"]
    chunk = c["degree"] - 2
    if sets:
        out.append((None, l_0 * (1 - sets[0][0]) % R))
        out.append((None, (sets[-1][0] * sets[-1][0] - sets[-1][0]) * l_last % R))
        for i in range(1, len(sets)):
            out.append((None, (sets[i][0] - sets[i - 1][2]) * l_0 % R))
        dlt = to_int(O.fr_const(5))
        for si, s in enumerate(sets):
            cols = c["perm_cols"][si * chunk:(si + 1) * chunk]
            sig = ev["perm_common"][si * chunk:(si + 1) * chunk]
            left = s[1]
            for (kind, ci), se in zip(cols, sig):
                e = col_eval(kind, ci)
                left = left * (e + beta * se + gamma) % R
            right = s[0]
            cur = beta * x % R * pow(dlt, si * chunk, R) % R
            for kind, ci in cols:
                e = col_eval(kind, ci)
                right = right * (e + cur + gamma) % R
                cur = cur * dlt % R
            out.append((None, (left - right) * (1 - (l_last + l_blind)) % R))
    # lookups: the boundary, one helper constraint per chunk, the accumulator
    for li, lk in enumerate(c["lookups"]):
        m, hs, Z, Zn = ev["lookups"][li]
        _, tab = lookup_columns(lk)
        table = 0
        for col in tab:
            table = (table * theta + fq(col)) % R
        sel = fq(lk["selector"]) if lk["selector"] is not None else 1
        out.append((None, (l_0 + l_last) * Z % R))
        for chunk, h in zip(lookup_chunks(c, lk), hs):
            fb = []
            for tup in chunk:
                f = 0
                for el in tup:
                    f = (f * theta + lookup_input_at(el)) % R
                fb.append((f + beta) % R)
            product, spp = 1, 0
            for j in range(len(fb)):
                partial = 1
                for i in range(len(fb)):
                    if i != j:
                        partial = partial * fb[i] % R
                spp += partial
                product = product * fb[j] % R
            out.append((None, (h * product - spp) % R))
        out.append((None, ((Zn - Z - sel * sum(hs)) * (table + beta) + m) * (1 - (l_last + l_blind)) % R))
    # trashcans (trash.rs:60-86): compressed - (1 - q) trash
    for ti, tc in enumerate(c.get("trashcans", [])):
        def read(col_type, col, rot):
            qs = (c["fixed_queries"], c["advice_queries"], c.get("instance_queries", []))[col_type]
            return (fix, adv, ins)[col_type][query_index(qs, col, rot)]
        compressed = program_at(tc["program"], read, ch)
        out.append((None, (compressed - (1 - fq(tc["selector"])) * ev["trash"][ti]) % R))
    return [(sel, v % R) for sel, v in out]


def program_at(graph, read, ch, all_values=False):
    """A flattened program (FlatGraphEvaluator, evaluation.rs:148-213) at one
    point with Python integers: each read is read(col_type, column, rotation)
    (the query's evaluation at x), the previous value zero, the challenge
    slots from ch; returns the result value.  partially_evaluate_identities
    evaluates the same gate expressions at x (plonk/mod.rs:537-562)."""
    vals = [0] * graph["values_len"]
    for i, cst in enumerate(graph["constants"]):
        vals[i] = to_int(cst)
    for slot, name in (("beta_idx", "beta"), ("theta_idx", "theta"), ("trash_challenge_idx", "trash"),
                       ("y_idx", "y")):
        vals[graph[slot]] = ch[name]
    vals[graph["previous_value_idx"]] = 0
    for t, col, r, dst in graph["reads"]:
        vals[dst] = read(t, col, graph["rotations"][r])
    for kind, dst, a, b, c in graph["ops"]:
        x, y2, z = vals[a], vals[b], vals[c]
        vals[dst] = [x + y2, x - y2, x * y2, x * x, 2 * x, -x, x * y2 + z][kind] % R
    return vals if all_values else vals[graph["result_idx"]]


def simple_selectors(circuit):
    """The fixed columns of simple selectors (ConstraintSystem::
    has_simple_selector_col): the selectors of the listed gate polynomials."""
    return {sel for _, sel in circuit.get("gate_polys", []) if sel is not None}


def linearization_split(tagged, y):
    """compute_linearization_poly's split (linearization/prover.rs:41-86):
    identity j of M gets y^(M-1-j); the untagged ones sum to the constant C,
    a tagged one scales its simple selector's fixed polynomial.  Returns
    (C, [(fixed column, coefficient)])."""
    c, terms, pw = 0, [], 1
    for sel, v in reversed(tagged):
        if sel is None:
            c = (c + pw * v) % R
        else:
            terms.append((sel, pw * v % R))
        pw = pw * y % R
    return c, terms


def horner(values, y):
    acc = 0
    for v in values:
        acc = (acc * y + v) % R
    return acc


# ---------------------------------------------------------- multi-open sets --
def intermediate_sets(queries):
    """construct_intermediate_sets (kzg/utils.rs:46-140): queries
    [(label, point)] -> (commitment labels in first-seen order with their set
    index, point sets as lists of points ordered by first-seen point index)."""
    point_index = {}
    com = []          # [label, [point indices]]
    for label, pt in queries:
        pi = point_index.setdefault(pt, len(point_index))
        for entry in com:
            if entry[0] == label:
                if pi in entry[1]:
                    raise ValueError("duplicated query")
                entry[1].append(pi)
                break
        else:
            com.append([label, [pi]])
    set_index = {}
    labels = []
    for label, pis in com:
        key = tuple(sorted(pis))
        si = set_index.setdefault(key, len(set_index))
        labels.append((label, si, key))
    inv_point = {i: p for p, i in point_index.items()}
    point_sets = [None] * len(set_index)
    for key, si in set_index.items():
        point_sets[si] = [inv_point[i] for i in key]
    return labels, point_sets, point_index


# ---------------------------------------------------------------- prover --
def instance_columns(key, instances):
    """compute_instances (prover.rs:475-539) without committed instances:
    each column's values zero-padded to n (Lagrange form); more values than
    usable rows is Error::InstanceTooLarge."""
    c, n = key.circuit, key.n
    instances = list(instances or [])
    if len(instances) != c.get("n_instance", 0):
        raise ValueError("wrong number of instance columns")
    cols = []
    for vals in instances:
        vals = np.ascontiguousarray(vals, np.uint64).reshape(-1, 4)
        if vals.shape[0] > key.u:
            raise ValueError("instance too large")
        col = np.zeros((n, 4), np.uint64)
        col[:vals.shape[0]] = vals
        cols.append(col)
    return instances, cols


def absorb_instances(tr, instances):
    """The transcript part of compute_instances: each column's length, then
    its values (common, prover.rs:503-512; verifier.rs:61-66)."""
    for vals in instances:
        vals = np.ascontiguousarray(vals, np.uint64).reshape(-1, 4)
        tr.common_fr(vals.shape[0])
        for v in vals:
            tr.common_fr(to_int(v))


def create_proof(key, advice, blinds, instances=None):
    """create_proof (plonk/prover.rs:432-473): compute_trace, then
    finalise_proof with the KZG multi_open (kzg/mod.rs:110-289).  advice:
    Lagrange values of every advice column (rows at and after the usable
    rows are replaced by blinding values); blinds: integers in the draw order
    of the module doc; instances: the values of each instance column.
    Returns the proof bytes."""
    c, dom, srs = key.circuit, key.dom, key.srs
    n, u, bf, qdeg = key.n, key.u, key.bf, key.qdeg
    blinds = list(blinds)
    if len(blinds) != blind_count(c):
        raise ValueError("wrong number of blinding values")
    bl = iter(blinds)
    take = lambda m: [next(bl) for _ in range(m)]
    instances, inst = instance_columns(key, instances)
    tr = Transcript()
    tr.common_fr(key.repr)                                    # vk.hash_into (prover.rs:101)
    absorb_instances(tr, instances)
    # parse_advices (prover.rs:541-632)
    adv = []
    for col in advice:
        a = np.ascontiguousarray(col, np.uint64).copy()
        a[u:] = np.stack([to_mont(v) for v in take(bf + 1)])
        adv.append(a)
    for a in adv:
        tr.write_point(commit(a, srs["lagrange"]))
    theta = tr.squeeze()
    # multiplicities (logup/prover.rs:95-184), committed in delta form
    ms, fs, ts = [], [], []
    # the input expressions over the Lagrange rows (compute_multiplicities_parallel)
    ex_lag = {pos: trash_column(key, g, adv, inst, 0, theta, 0) for pos, g in lookup_exprs(c)}
    for li, lk in enumerate(c["lookups"]):
        sel = key.fixed_values[lk["selector"]] if lk["selector"] is not None else np.tile(O.fr_const(0), (n, 1))
        ins, tab = lookup_columns(lk)
        col = lambda ti, ei, el: adv[el] if is_column(el) else ex_lag[(li, ti, ei)]
        fl = [col(ti, 0, tup[0]) if len(tup) == 1 else compress_columns([col(ti, ei, el) for ei, el in enumerate(tup)],
                                                                         theta) for ti, tup in enumerate(ins)]
        t = key.fixed_values[tab[0]] if len(tab) == 1 else compress_columns([key.fixed_values[i] for i in tab], theta)
        ms.append(compute_multiplicities(sel, fl, t, u, take(bf + 1)))
        fs.append(fl)
        ts.append(t)
    for m in ms:
        tr.write_point(commit(delta(m, 1), srs["delta"]))
    beta = tr.squeeze()
    gamma = tr.squeeze()
    S = n_perm_sets(c)
    perm_bl = [take(bf) for _ in range(S)]
    log_bl = [take(bf) for _ in c["lookups"]]
    # permutation products (permutation/prover.rs:81-255) and logup helper / aggregator
    pvals = [(adv, key.fixed_values, inst)[kind][ci] for kind, ci in c["perm_cols"]]
    zs = O.permutation_z(pvals, key.perm_values, c["degree"] - 2, c["k"], to_mont(key.omega), to_mont(beta),
                         to_mont(gamma), bf, np.stack([np.stack([to_mont(v) for v in b]) for b in perm_bl])) if S else []
    hs, Zs = [], []   # hs: per lookup, its helpers (one per chunk of inputs)
    for li, lk in enumerate(c["lookups"]):
        sel = key.fixed_values[lk["selector"]] if lk["selector"] is not None else np.tile(O.fr_const(0), (n, 1))
        per = lookup_per_helper(c, lk)
        chunks = [fs[li][i:i + per] for i in range(0, len(fs[li]), per)]
        hl, Z = O.logup(chunks, ts[li], sel, ms[li], to_mont(beta), bf, np.stack([to_mont(v) for v in log_bl[li]]))
        hs.append(list(hl))
        Zs.append(Z)
    for z in zs:
        tr.write_point(commit(delta(z, 1), srs["delta"]))
    for hl, Z in zip(hs, Zs):                                  # prover.rs:221-227
        for h in hl:
            tr.write_point(commit(h, srs["lagrange"]))
        tr.write_point(commit(delta(Z, 2), srs["double_delta"]))
    trash = tr.squeeze()
    # trash columns (trash/prover.rs:29-77): the constraint expressions over
    # the Lagrange columns, compressed with the trash challenge
    trs = [trash_column(key, tc["program"], adv, inst, beta, theta, trash) for tc in c.get("trashcans", [])]
    for t in trs:
        tr.write_point(commit(t, srs["lagrange"]))
    y = tr.squeeze()
    # coefficient forms and cosets
    adv_c = [dom.lagrange_to_coeff(a) for a in adv]
    z_c = [dom.lagrange_to_coeff(z) for z in zs]
    m_c = [dom.lagrange_to_coeff(m) for m in ms]
    h_c = [[dom.lagrange_to_coeff(h) for h in hl] for hl in hs]
    Z_c = [dom.lagrange_to_coeff(Z) for Z in Zs]
    ext = lambda p: dom.coeff_to_extended(p)
    inst_c = [dom.lagrange_to_coeff(col) for col in inst]
    t_c = [dom.lagrange_to_coeff(t) for t in trs]
    hpoly = quotient(key, [ext(p) for p in adv_c], [ext(p) for p in z_c], [ext(p) for p in m_c],
                     [[ext(p) for p in hl] for hl in h_c], [ext(p) for p in Z_c], y, beta, gamma, theta, trash=trash,
                     inst_e=[ext(p) for p in inst_c], trash_e=[ext(p) for p in t_c])
    hcoeff = dom.extended_to_coeff(hpoly)[: (n - 1) * qdeg]
    limbs = [np.concatenate([hcoeff[i * (n - 1):(i + 1) * (n - 1)], np.zeros((1, 4), np.uint64)]) for i in range(qdeg)]
    for i, t in enumerate(take(qdeg - 1), start=1):         # blind_quotient_limbs (prover.rs:774-785)
        limbs[i - 1][n - 1] = to_mont(t)
        limbs[i][0] = to_mont(to_int(limbs[i][0]) - t)
    for lb in limbs:
        tr.write_point(commit(lb, srs["g"]))
    x = tr.squeeze()
    xn = pow(x, n, R)
    # evaluations (prover.rs:798-868, permutation/prover.rs:270-335, logup/prover.rs:318-352)
    simple = simple_selectors(c)
    ev = {"advice": [eval_at(adv_c[col], rotate(key, x, rot)) for col, rot in c["advice_queries"]],
          "fixed": [1 if col in simple else eval_at(key.fixed_polys[col], rotate(key, x, rot))
                    for col, rot in c["fixed_queries"]]}
    for v in ev["advice"]:
        tr.write_fr(v)
    for (col, _), v in zip(c["fixed_queries"], ev["fixed"]):
        if col not in simple:                                  # a simple selector's is not written
            tr.write_fr(v)
    ev["perm_common"] = [eval_at(p, x) for p in key.perm_polys]
    for v in ev["perm_common"]:
        tr.write_fr(v)
    x_next, x_last = rotate(key, x, 1), rotate(key, x, -(bf + 1))
    sets = []
    for si, z in enumerate(z_c):
        s = [eval_at(z, x), eval_at(z, x_next), eval_at(z, x_last) if si < S - 1 else None]
        sets.append(s)
        tr.write_fr(s[0])
        tr.write_fr(s[1])
        if s[2] is not None:
            tr.write_fr(s[2])
    ev["perm_sets"] = sets
    ev["lookups"] = []
    for li in range(len(c["lookups"])):
        e = (eval_at(m_c[li], x), [eval_at(h, x) for h in h_c[li]], eval_at(Z_c[li], x), eval_at(Z_c[li], x_next))
        ev["lookups"].append(e)
        for v in (e[0], *e[1], e[2], e[3]):
            tr.write_fr(v)
    ev["trash"] = [eval_at(t, x) for t in t_c]                 # trash/prover.rs:80-92
    for v in ev["trash"]:
        tr.write_fr(v)
    # linearization (linearization/prover.rs:41-86): L'(X) = sum over the
    # identities with a simple selector of y^(M-1-j) id_j(x) S_j(X), minus
    # sum_i (x^n - 1) (x^(n-1))^i h_i(X)
    sf = pow(x, n - 1, R)
    polys = list(limbs)
    coefs = [to_mont(-(xn - 1) * pow(sf, i, R)) for i in range(qdeg)]
    if simple:
        ev["instance"] = [eval_at(inst_c[col], rotate(key, x, rot)) for col, rot in c.get("instance_queries", [])]
        ch = {"x": x, "xn": xn, "beta": beta, "gamma": gamma, "theta": theta, "trash": trash, "y": y}
        _, terms = linearization_split(identities(key, ev, ch), y)
        for sel, v in terms:
            polys.append(key.fixed_polys[sel])
            coefs.append(to_mont(v))
    lin = O.poly_inner_product(polys, coefs)
    # queries (prover.rs:871-933)
    q = []
    for col, rot in c["advice_queries"]:
        q.append((("advice", col), rotate(key, x, rot), adv_c[col]))
    for si, z in enumerate(z_c):
        q.append((("perm", si), x, z))
        q.append((("perm", si), x_next, z))
    for si in reversed(range(S - 1)):
        q.append((("perm", si), x_last, z_c[si]))
    for li in range(len(c["lookups"])):
        q.append((("m", li), x, m_c[li]))
        for j, h in enumerate(h_c[li]):
            q.append((("h", li, j), x, h))
        q.append((("Z", li), x, Z_c[li]))
        q.append((("Z", li), x_next, Z_c[li]))
    for ti, t in enumerate(t_c):
        q.append((("trash", ti), x, t))
    for col, rot in c["fixed_queries"]:
        if col not in simple:                                  # prover.rs:913-918
            q.append((("fixed", col), rotate(key, x, rot), key.fixed_polys[col]))
    for i, p in enumerate(key.perm_polys):
        q.append((("perm_fixed", i), x, p))
    q.append((("lin",), x, lin))
    multi_open(key, tr, q)
    return bytes(tr.proof)


def trash_column(key, graph, adv, inst, beta, theta, trash):
    """Argument::commit's compressed expression (trash/prover.rs:46-62): the
    program (the constraint expressions folded with the trash challenge) at
    every row of the n-point domain over the Lagrange columns, rotations in
    rows.  Pure Python per row: small domains."""
    n = key.n
    cols = (key.fixed_values, adv, inst)
    ch = (to_mont(beta), to_mont(theta), to_mont(trash), np.zeros(4, np.uint64))
    out = np.zeros((n, 4), np.uint64)
    for r in range(n):
        out[r] = O._run_program(graph, cols, r, n, 0, ch)[graph["result_idx"]]
    return out


def quotient(key, adv_e, z_e, m_e, h_e, Z_e, y, beta, gamma, theta, threads=None, trash=0, inst_e=(), trash_e=()):
    """compute_nu_poly + divide_by_vanishing_poly (prover.rs:634-715) through
    the C oracle's evaluate_numerator restatement."""
    c, dom = key.circuit, key.dom
    keep = []

    def parr(items):
        arr = (O.ctypes.c_void_p * max(1, len(items)))(*[a.ctypes.data for a in items])
        keep.append(arr)
        return O.ctypes.cast(arr, O.ctypes.POINTER(O.ctypes.c_void_p))

    def u32(items):
        arr = (O.ctypes.c_uint32 * max(1, len(items)))(*items)
        keep.append(arr)
        return O.ctypes.cast(arr, O.ctypes.POINTER(O.ctypes.c_uint32))

    d = O.QuotientDesc()
    d.k, d.extended_k = c["k"], dom.extended_k
    d.advice, d.n_advice = parr(adv_e), len(adv_e)
    d.fixed, d.n_fixed = parr(key.fixed_cosets), len(key.fixed_cosets)
    d.gate_fixed[:] = c.get("gate_fixed", [0] * 5)
    d.gate_advice[:] = c.get("gate_advice", [0] * 3)
    d.n_perm_cols = len(c["perm_cols"])
    d.perm_col_kind = u32([kind for kind, _ in c["perm_cols"]])
    d.perm_col_index = u32([ci for _, ci in c["perm_cols"]])
    d.perm_sigma = parr(key.perm_cosets)
    d.n_perm_sets, d.perm_z = len(z_e), parr(z_e)
    d.chunk_len, d.blinding_factors = c["degree"] - 2, key.bf
    tcs = c.get("trashcans", [])
    shapes = [lookup_columns(lk) for lk in c["lookups"]]
    builtin = (len(shapes) == 1 and not tcs and len(shapes[0][0]) == 1 and len(shapes[0][1]) == 1
               and is_column(shapes[0][0][0][0]))
    if builtin:
        lk = c["lookups"][0]
        d.has_lookup = 1
        d.lookup_input_advice, d.lookup_table_fixed = shapes[0][0][0][0], shapes[0][1][0]
        d.lookup_selector_fixed = -1 if lk["selector"] is None else lk["selector"]
        d.lookup_h, d.lookup_z, d.lookup_m = h_e[0][0].ctypes.data, Z_e[0].ctypes.data, m_e[0].ctypes.data
    d.l0, d.l_last, d.l_active = key.l0.ctypes.data, key.l_last.ctypes.data, key.l_active.ctypes.data
    for name, v in (("y", y), ("beta", beta), ("gamma", gamma), ("theta", theta)):
        getattr(d, name)[:] = [int(t) for t in to_mont(v)]
    d.extended_omega[:] = [int(t) for t in dom.get(2)]
    d.g_coset[:] = [int(t) for t in dom.get(3)]
    inst_e = list(inst_e)
    d.instance, d.n_instance = parr(inst_e), len(inst_e)
    keep.extend([adv_e, z_e, m_e, h_e, Z_e, inst_e])
    gate_values = None
    if c.get("gates") is not None:
        gate_values = O.flat_gates_eval(c["gates"], key.fixed_cosets, adv_e, inst_e, c["k"], dom.extended_k,
                                        to_mont(beta), to_mont(theta), to_mont(trash), to_mont(y))
    if builtin or (not c["lookups"] and not tcs):
        return dom.quotient_eval(d, True, threads, gate_values)
    # several lookups, tuples, parallel inputs or trashcans: the gate and
    # permutation terms, then every lookup's terms (evaluation.rs:1034-1090)
    # as one helper program per chunk (Evaluator::lookups_flat, :691-770) and
    # every trashcan's term (:1093-1109), then the division by t(X)
    v = dom.quotient_eval(d, False, threads, gate_values)
    # the input expressions on the extended coset, read as advice columns
    # after the circuit's
    zero = np.zeros(4, np.uint64)
    exprs = lookup_exprs(c)
    ex_e = [O.flat_gates_eval(g, key.fixed_cosets, adv_e, inst_e, c["k"], dom.extended_k, zero, to_mont(theta), zero,
                              zero) for _, g in exprs]
    ex_col = {pos: len(adv_e) + j for j, (pos, _) in enumerate(exprs)}
    lks = []
    for li, lk in enumerate(c["lookups"]):
        per = lookup_per_helper(c, lk)
        col = lambda ti, ei, el: el if is_column(el) else ex_col[(li, ti, ei)]
        progs = [lookup_program(lk, chunk, first=j == 0, col=col, t0=j * per)
                 for j, chunk in enumerate(lookup_chunks(c, lk))]
        lks.append({"programs": [g for g, _ in progs], "outputs": [o for _, o in progs], "helpers": list(h_e[li]),
                    "aggregator": Z_e[li], "multiplicities": m_e[li]})
    tas = [{"program": tc["program"], "selector": tc["selector"], "trash": trash_e[ti]} for ti, tc in enumerate(tcs)]
    v = O.flat_tail_eval(v, key.fixed_cosets, list(adv_e) + ex_e, inst_e, c["k"], dom.extended_k, to_mont(beta), to_mont(theta),
                         to_mont(trash), to_mont(y), key.l0, key.l_last, key.l_active, lookups=lks, trashcans=tas)
    return dom.divide_by_vanishing_poly(v)


def lookup_columns(lk):
    """(input tuples, table tuple) of a lookup: "input" one advice column or
    a tuple (list) of them, or "inputs" a list of such tuples (parallel
    lookups into one table, BatchedArgument::new, logup.rs:226-262); "table"
    one fixed column or a tuple of the inputs' width."""
    one = lambda v: list(v) if isinstance(v, (list, tuple)) else [v]
    ins = [one(t) for t in lk["inputs"]] if "inputs" in lk else [one(lk["input"])]
    return ins, one(lk["table"])


def is_column(el):
    """A lookup input element that is an advice column (else an expression)."""
    return isinstance(el, (int, np.integer))


def program_degree(graph):
    """Expression::degree (plonk/circuit.rs:1074-1086) of a program's result:
    a column read 1, a constant or challenge slot 0, a product the sum of its
    factors' degrees, a sum the larger one."""
    deg = [0] * graph["values_len"]
    for _, _, _, dst in graph["reads"]:
        deg[dst] = 1
    for kind, dst, a, b, cc in graph["ops"]:
        deg[dst] = (max(deg[a], deg[b]) if kind in (0, 1) else deg[a] + deg[b] if kind == 2 else
                    2 * deg[a] if kind == 3 else deg[a] if kind in (4, 5) else max(deg[a] + deg[b], deg[cc]))
    return deg[graph["result_idx"]]


def lookup_exprs(circuit):
    """The lookup input elements that are expressions, in order (lookup,
    input tuple, element): [((lookup, tuple, element), program)]."""
    out = []
    for li, lk in enumerate(circuit["lookups"]):
        for ti, tup in enumerate(lookup_columns(lk)[0]):
            out.extend(((li, ti, ei), el) for ei, el in enumerate(tup) if not is_column(el))
    return out


def lookup_per_helper(circuit, lk=None):
    """Parallel inputs per helper polynomial (nb_parallel_lookups_per_chunk,
    logup.rs:168-183): next_pow2(cs.degree() - 1) over the largest degree
    of the lookup's input expressions (1 for columns)."""
    p = 1
    while p < circuit["degree"] - 1:
        p *= 2
    d = 1
    if lk is not None:
        d = max(1 if is_column(el) else program_degree(el) for tup in lookup_columns(lk)[0] for el in tup)
    return p // d


def lookup_chunks(circuit, lk):
    """The lookup's input tuples split into helper chunks
    (chunk_by_degree, logup.rs:289-300)."""
    ins, _ = lookup_columns(lk)
    per = lookup_per_helper(circuit, lk)
    return [ins[i:i + per] for i in range(0, len(ins), per)]


def compress_columns(cols, theta):
    """The theta-compression of a tuple of columns (compress_expressions:
    Horner in the tuple's order, the first column times theta^(w-1))."""
    w = len(cols)
    return O.poly_inner_product(list(cols), [to_mont(pow(theta, w - 1 - e, R)) for e in range(w)])


def lookup_program(lk, chunk, first=True, col=lambda ti, ei, el: el, t0=0):
    """The helper program of one chunk of a lookup's input tuples
    (Evaluator::lookups_flat, evaluation.rs:691-770): values 0, 1
    (constants), beta, theta, trash challenge, y, the previous value, the
    reads; every input tuple theta-compressed (Horner from 0 theta + the
    first column) plus beta, f_j; the product of the f_j and the sum of
    partial products sum_j prod_{i!=j} f_i (each by a loop over i, as the
    reference builds it; one input: the constant one); for the first chunk
    the compressed table plus beta and the selector.  col(tuple, element,
    input) gives the advice column a read takes (an expression input's
    values sit in an extra column), t0 the index of the chunk's first tuple.
    Returns (graph, (sum_partial_products, product, table, selector)
    indices)."""
    _, tab = lookup_columns(lk)
    reads, ops = [], []
    slot = [7]

    def new():
        slot[0] += 1
        return slot[0] - 1

    def op(kind, a, b, cc=0):
        d = new()
        ops.append((kind, d, a, b, cc))
        return d
    in_at = [[None] * len(tup) for tup in chunk]
    for j, tup in enumerate(chunk):
        for e, el in enumerate(tup):
            in_at[j][e] = new()
            reads.append((1, col(t0 + j, e, el), 0, in_at[j][e]))
    table = sel = 1
    if first:
        tab_at = []
        for tcol in tab:
            tab_at.append(new())
            reads.append((0, tcol, 0, tab_at[-1]))
        if lk["selector"] is not None:
            sel = new()
            reads.append((0, lk["selector"], 0, sel))
    f = []
    for j in range(len(chunk)):
        acc = 0
        for e in range(len(chunk[j])):
            acc = op(6, acc, 3, in_at[j][e])
        f.append(op(0, acc, 2))
    if first:
        acc = 0
        for t in tab_at:
            acc = op(6, acc, 3, t)
        table = op(0, acc, 2)
    product, spp = f[0], 1
    if len(f) > 1:
        partials = []
        for j in range(len(f)):
            acc = 1
            for i in range(len(f)):
                if i != j:
                    acc = op(2, acc, f[i])
            partials.append(acc)
        spp = partials[0]
        for pj in partials[1:]:
            spp = op(0, spp, pj)
        product = f[0]
        for fj in f[1:]:
            product = op(2, product, fj)
    graph = {"constants": [np.zeros(4, np.uint64), O.fr_const(0)], "rotations": [0], "reads": reads, "ops": ops,
             "values_len": slot[0], "beta_idx": 2, "theta_idx": 3, "trash_challenge_idx": 4, "y_idx": 5,
             "previous_value_idx": 6, "result_idx": spp}
    return graph, (spp, product, table, sel)


def multi_open(key, tr, queries):
    """KZGCommitmentScheme::multi_open (kzg/mod.rs:110-289) without the
    fewer-point-sets and truncated-challenges features."""
    srs = key.srs
    x1 = tr.squeeze()
    x2 = tr.squeeze()
    label_poly = {}
    for label, _, poly in queries:
        label_poly[label] = poly
    labels, point_sets, _ = intermediate_sets([(lb, pt) for lb, pt, _ in queries])
    per_set = [[] for _ in point_sets]
    for label, si, _ in labels:
        per_set[si].append(label_poly[label])
    q_polys = [O.poly_inner_product(ps, [to_mont(v) for v in powers(x1, len(ps))]) for ps in per_set]
    order = sorted(range(len(point_sets)), key=lambda i: (len(point_sets[i]), i))
    q_polys = [q_polys[i] for i in order]
    point_sets = [point_sets[i] for i in order]
    f_polys = []
    for pts, qp in zip(point_sets, q_polys):
        p = qp
        for pt in pts:
            p = O.kate_division(p, to_mont(pt))
        f_polys.append(p)
    f = O.poly_inner_product(f_polys, [to_mont(v) for v in powers(x2, len(f_polys))])
    tr.write_point(commit(f, srs["g"]))
    x3 = tr.squeeze()
    for qp in q_polys:
        tr.write_fr(eval_at(qp, x3))
    x4 = tr.squeeze()
    final = O.poly_inner_product(q_polys + [f], [to_mont(v) for v in powers(x4, len(q_polys) + 1)])
    v = eval_at(final, x3)
    final = final.copy()
    final[0] = to_mont(to_int(final[0]) - v)
    tr.write_point(commit(O.kate_division(final, to_mont(x3)), srs["g"]))


# --------------------------------------------------------------- verifier --
def verify(key, proof, s_trapdoor, instances=None):
    """prepare (plonk/verifier.rs:371-407: parse_trace, then
    verify_algebraic_constraints) and KZGCommitmentScheme::multi_prepare
    (kzg/mod.rs:291-491), finished by DualMSM::check (kzg/msm.rs:294-310)
    with the pairing e(pi, [s]G2) = e(C - vG + x3 pi, G2) replaced by the
    equivalent G1 check [s]pi = C - vG + x3 pi for the test setup's known s.
    The instance columns' values are absorbed as the prover absorbs them
    and their evaluations computed from the values (verifier.rs:205-242).
    Returns True or False; a malformed proof is False."""
    try:
        return _verify(key, proof, s_trapdoor, instances)
    except ValueError:
        return False


def _verify(key, proof, s, instances=None):
    c = key.circuit
    n, bf, qdeg = key.n, key.bf, key.qdeg
    S = n_perm_sets(c)
    L = len(c["lookups"])
    instances, _ = instance_columns(key, instances)
    tr = Transcript(proof)
    tr.common_fr(key.repr)
    absorb_instances(tr, instances)
    adv_coms = [tr.read_point() for _ in range(c["n_advice"])]
    theta = tr.squeeze()
    m_coms = [tr.read_point() for _ in range(L)]
    beta = tr.squeeze()
    gamma = tr.squeeze()
    z_coms = [tr.read_point() for _ in range(S)]
    hz_coms = []   # per lookup: (its helpers' commitments, its aggregator's)
    for lk in c["lookups"]:
        hl = [tr.read_point() for _ in lookup_chunks(c, lk)]
        hz_coms.append((hl, tr.read_point()))
    trash = tr.squeeze()
    T = len(c.get("trashcans", []))
    trash_coms = [tr.read_point() for _ in range(T)]
    y = tr.squeeze()
    limb_coms = [tr.read_point() for _ in range(qdeg)]
    x = tr.squeeze()
    sf = pow(x, n - 1, R)
    xn = sf * x % R
    simple = simple_selectors(c)
    ev = {"advice": [tr.read_fr() for _ in c["advice_queries"]],
          "fixed": [1 if col in simple else tr.read_fr() for col, _ in c["fixed_queries"]]}
    ev["perm_common"] = [tr.read_fr() for _ in c["perm_cols"]]
    sets = []
    for si in range(S):
        z0, z1 = tr.read_fr(), tr.read_fr()
        sets.append([z0, z1, tr.read_fr() if si < S - 1 else None])
    ev["perm_sets"] = sets
    ev["lookups"] = [(tr.read_fr(), [tr.read_fr() for _ in lookup_chunks(c, lk)], tr.read_fr(), tr.read_fr())
                     for lk in c["lookups"]]
    ev["trash"] = [tr.read_fr() for _ in range(T)]
    ev["instance"] = instance_evals(key, instances, x, xn)
    ch = {"x": x, "xn": xn, "beta": beta, "gamma": gamma, "theta": theta, "trash": trash, "y": y}
    const, terms = linearization_split(identities(key, ev, ch), y)
    # compute_linearization_commitment (linearization/verifier.rs:27-78)
    lin_com = pt_lincomb(limb_coms + [key.fixed_coms[sel] for sel, _ in terms],
                         [(1 - xn) * pow(sf, i, R) for i in range(qdeg)] + [v for _, v in terms])
    lin_eval = -const % R
    x_next, x_last = rotate(key, x, 1), rotate(key, x, -(bf + 1))
    q = []   # (label, point, commitment, eval)
    for qi, (col, rot) in enumerate(c["advice_queries"]):
        q.append((("advice", col), rotate(key, x, rot), adv_coms[col], ev["advice"][qi]))
    for si in range(S):
        q.append((("perm", si), x, z_coms[si], sets[si][0]))
        q.append((("perm", si), x_next, z_coms[si], sets[si][1]))
    for si in reversed(range(S - 1)):
        q.append((("perm", si), x_last, z_coms[si], sets[si][2]))
    for li in range(L):
        m, hs, Z, Zn = ev["lookups"][li]
        q.append((("m", li), x, m_coms[li], m))
        for j, h in enumerate(hs):
            q.append((("h", li, j), x, hz_coms[li][0][j], h))
        q.append((("Z", li), x, hz_coms[li][1], Z))
        q.append((("Z", li), x_next, hz_coms[li][1], Zn))
    for ti in range(T):
        q.append((("trash", ti), x, trash_coms[ti], ev["trash"][ti]))
    for qi, (col, rot) in enumerate(c["fixed_queries"]):
        if col not in simple:
            q.append((("fixed", col), rotate(key, x, rot), key.fixed_coms[col], ev["fixed"][qi]))
    for i, com in enumerate(key.perm_coms):
        q.append((("perm_fixed", i), x, com, ev["perm_common"][i]))
    q.append((("lin",), x, lin_com, lin_eval))
    # multi_prepare
    x1 = tr.squeeze()
    x2 = tr.squeeze()
    label_com = {lb: com for lb, _, com, _ in q}
    labels, point_sets, point_index = intermediate_sets([(lb, pt) for lb, pt, _, _ in q])
    evals_of = {}
    for lb, pt, _, e in q:
        evals_of.setdefault(lb, {})[pt] = e
    q_coms = [[] for _ in point_sets]
    q_evals = [[] for _ in point_sets]
    for label, si, _ in labels:
        q_coms[si].append(label_com[label])
        q_evals[si].append([evals_of[label][pt] for pt in point_sets[si]])
    nb = max(len(v) for v in q_coms)
    px1 = powers(x1, nb)
    q_com = [pt_lincomb(coms, px1) for coms in q_coms]
    q_ev = [[sum(px1[j] * ev_j[i] for j, ev_j in enumerate(evs)) % R for i in range(len(evs[0]))] for evs in q_evals]
    order = sorted(range(len(point_sets)), key=lambda i: (len(point_sets[i]), i))
    q_com = [q_com[i] for i in order]
    q_ev = [q_ev[i] for i in order]
    point_sets = [point_sets[i] for i in order]
    f_com = tr.read_point()
    x3 = tr.squeeze()
    q_x3 = [tr.read_fr() for _ in point_sets]
    f_eval = 0
    for pts, evs, pe in reversed(list(zip(point_sets, q_ev, q_x3))):
        r_eval = lagrange_eval(pts, evs, x3)
        den = 1
        for p in pts:
            den = den * (x3 - p) % R
        f_eval = (f_eval * x2 + (pe - r_eval) * inv(den)) % R
    x4 = tr.squeeze()
    p4 = powers(x4, len(q_com) + 1)
    final_com = pt_lincomb(q_com + [f_com], p4)
    v = sum(a * b for a, b in zip(q_x3 + [f_eval], p4)) % R
    pi = tr.read_point()
    tr.assert_empty()
    gen = O.g1_generator()
    right = pt_add(pt_add(final_com, pt_mul(gen, -v % R)), pt_mul(pi, x3))
    return bool(np.array_equal(pt_mul(pi, s), right))


def lagrange_eval(points, evals, at):
    """The interpolating polynomial of (points, evals) evaluated at `at`
    (lagrange_interpolate, utils/arithmetic.rs:183-245, then eval_polynomial)."""
    total = 0
    for j, (xj, yj) in enumerate(zip(points, evals)):
        num, den = 1, 1
        for k2, xk in enumerate(points):
            if k2 != j:
                num = num * (at - xk) % R
                den = den * (xj - xk) % R
        total = (total + yj * num * inv(den)) % R
    return total
