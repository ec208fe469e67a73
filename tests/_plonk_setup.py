"""A config-3 circuit (the single-proof configuration) set up on the device
and in the oracle: seeded fixed columns, copy cycles and witness, the KZG
test SRS generated on the device (its bases are pinned against the oracle in
test_srs_gpu.py) and handed to the oracle, and both keys."""
import numpy as np

from _loader import load
from oracle import oracle as O
from oracle import plonk as OP

mzk = load()


# stands for format!("{:?}", domain.pinned()) + format!("{:?}", cs.pinned())
PINNED = b"config-3 circuit: standard gate, copy cycles, range lookup"


SHAPES = {"config3": (OP.config3_circuit, OP.config3_instance), "generic": (OP.generic_circuit, OP.generic_instance),
          "generic2": (OP.generic2_circuit, OP.generic2_instance),
          "instance": (OP.instance_circuit, OP.instance_instance),
          "trash": (OP.trash_circuit, OP.trash_instance),
          "selector": (OP.selector_circuit, OP.selector_instance),
          "tuple": (OP.tuple_circuit, OP.tuple_instance),
          "parallel": (OP.parallel_circuit, OP.parallel_instance),
          "nolookup": (OP.nolookup_circuit, OP.nolookup_instance),
          "bare": (OP.bare_circuit, OP.bare_instance),
          "expr": (OP.expr_circuit, OP.expr_instance),
          "many": (OP.many_circuit, OP.many_instance)}


class Circuit:
    def __init__(self, ctx, k, seed, pinned=PINNED, oracle=True, srs=None, shape="config3"):
        """srs = (buffer, offsets) of a shared device SRS whose bases hold this
        k's g | lagrange | delta | double delta at the offsets; otherwise
        this circuit gets its own.  shape: "config3" (the single-proof
        configuration), "generic" (two gates with a rotation, two
        permutation sets), "generic2" (generic with a second lookup,
        without a selector), "instance" (generic with an instance column
        read by a third gate and copied from c), "trash" (generic with a
        trashcan), "selector" (generic with a simple selector), "tuple"
        (generic with a lookup of the tuple (a, d) into (table, squares)) or
        "parallel" (lookups with parallel inputs: two helper chunks, and
        two tuples in one chunk), "nolookup" (generic without its lookup),
        "bare" (generic without lookup and permutation), "expr" (lookups
        whose inputs are expressions: a rotation, products) or "many" (five
        lookups and five trashcans)."""
        self.ctx, self.k, self.seed = ctx, k, seed
        make_circuit, make_instance = SHAPES[shape]
        c = make_circuit(k)
        c["blinding_factors"] = OP.blinding_factors(c)
        self.circuit = c
        made = make_instance(k, seed)
        self.fixed, self.mapping, self.advice = made[:3]
        self.instances = made[3] if len(made) > 3 else None
        self.dom = mzk.EvaluationDomain(ctx, c["degree"], k)
        n = self.n = self.dom.n
        if srs is None:
            self.s = O.rand_fr(1000 + seed, 1)[0]
            self.srs_buf = ctx.alloc(4 * n * 96)
            p = self.srs_buf.ptr
            self.dom.srs_setup_device(self.s, p, p + n * 96, p + 2 * n * 96, p + 3 * n * 96)
            self.offs = (0, n, 2 * n, 3 * n)
            self.desc = mzk.SrsDesc(p, 4 * n, 0, n, 2 * n, 3 * n, 0, 0, 0)
        else:
            self.srs_buf, self.offs, self.desc, self.s = srs
        self.key = mzk.PlonkKey(ctx, self.dom, c, self.desc, self.fixed, self.mapping, pinned)
        self.okey = None
        if oracle:
            host = self.srs_buf.download((self.desc.srs_len, 12))
            g, lag, dl, ddl = (host[o:o + n] for o in self.offs)
            srs_h = {"g": g, "lagrange": lag, "delta": dl, "double_delta": ddl}
            self.okey = OP.keygen(make_circuit(k), self.fixed, self.mapping, srs_h, pinned)

    def blinds(self, seed):
        return O.rand_fr(5000 + seed, self.key.n_blinds)

    def oracle_proof(self, advice, blinds, instances=None):
        return OP.create_proof(self.okey, advice, [OP.to_int(v) for v in blinds],
                               self.instances if instances is None else instances)

    def verify(self, proof, instances=None):
        return OP.verify(self.okey, proof, OP.to_int(self.s), self.instances if instances is None else instances)
