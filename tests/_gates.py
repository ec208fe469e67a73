"""A sample custom-gate program in the layout of the reference's flattened
evaluator (FlatGraphEvaluator, proofs/src/plonk/evaluation.rs:148-213):
values [constants | beta, theta, trash_challenge, y, previous_value | column
reads | intermediates].  Three gates over fixed f0..f2, advice a0..a2 and one
instance column i0, with rotations 0, +1, -1, every op kind, a constant and
a challenge read:
    g1 = f0 a0 a1(+1) + a2 - c0
    g2 = a1^2 - 2 a0(-1) f1
    g3 = -(a2 f2) + a0(+1) theta + i0
    result = ((prev y + g1) y + g2) y + g3          (Horner in y, prev = 0)
"""
ADD, SUB, MUL, SQUARE, DOUBLE, NEGATE, MULADD = range(7)
FIXED, ADVICE, INSTANCE = 0, 1, 2
BETA, THETA, TRASH, Y, PREV = 1, 2, 3, 4, 5

ROTATIONS = [0, 1, -1]
READS = [  # (col_type, col_idx, rot_idx, dst)
    (ADVICE, 0, 0, 6), (ADVICE, 1, 1, 7), (ADVICE, 2, 0, 8), (FIXED, 0, 0, 9), (ADVICE, 1, 0, 10),
    (ADVICE, 0, 2, 11), (FIXED, 1, 0, 12), (FIXED, 2, 0, 13), (ADVICE, 0, 1, 14), (INSTANCE, 0, 0, 15),
]
OPS = [  # (kind, dst, a, b, c)
    (MUL, 16, 9, 6, 0), (MUL, 17, 16, 7, 0), (ADD, 18, 17, 8, 0), (SUB, 19, 18, 0, 0),          # g1
    (SQUARE, 20, 10, 0, 0), (MUL, 21, 11, 12, 0), (DOUBLE, 22, 21, 0, 0), (SUB, 23, 20, 22, 0),  # g2
    (MUL, 24, 8, 13, 0), (NEGATE, 25, 24, 0, 0), (MUL, 26, 14, THETA, 0), (ADD, 27, 25, 26, 0),
    (ADD, 28, 27, 15, 0),                                                                       # g3
    (MULADD, 29, PREV, Y, 19), (MULADD, 30, 29, Y, 23), (MULADD, 31, 30, Y, 28),                 # Horner
]
VALUES_LEN, RESULT = 32, 31


def sample_graph(c0):
    """The program as the dict the oracle's flat_gates_eval takes."""
    return {"constants": [c0], "rotations": ROTATIONS, "reads": READS, "ops": OPS, "values_len": VALUES_LEN,
            "beta_idx": BETA, "theta_idx": THETA, "trash_challenge_idx": TRASH, "y_idx": Y,
            "previous_value_idx": PREV, "result_idx": RESULT}


def standard_gate_graph():
    """q_l a + q_r b + q_m a b + q_o c + q_c (fixed 0..4, advice 0..2) as a
    program: the standard gate of the fused kernel."""
    reads = [(FIXED, i, 0, 6 + i) for i in range(5)] + [(ADVICE, i, 0, 11 + i) for i in range(3)]
    ops = [(MUL, 14, 6, 11), (MUL, 15, 7, 12), (ADD, 16, 14, 15), (MUL, 17, 11, 12), (MUL, 18, 17, 8),
           (ADD, 19, 16, 18), (MUL, 20, 9, 13), (ADD, 21, 19, 20), (ADD, 22, 21, 10), (MULADD, 23, PREV, Y, 22)]
    return {"constants": [], "rotations": [0], "reads": reads, "ops": [o + (0,) * (5 - len(o)) for o in ops],
            "values_len": 24, "beta_idx": BETA, "theta_idx": THETA, "trash_challenge_idx": TRASH, "y_idx": Y,
            "previous_value_idx": PREV, "result_idx": 23}


def single_lookup_graph(input_advice, table_fixed, selector_fixed):
    """The built-in lookup of the fused kernel as a helper program: one input
    expression (a single advice column) compressed with theta, so
    product = a + beta, sum of partial products = 1 (Store(Constant(1)) of
    the reference for one input, evaluation.rs:730-740), table = t + beta,
    selector = s.  Constants [0, 1] as GraphEvaluator's first constants.
    Returns (graph, outputs)."""
    reads = [(ADVICE, input_advice, 0, 7), (FIXED, table_fixed, 0, 8), (FIXED, selector_fixed, 0, 9)]
    ops = [(MULADD, 10, 0, 3, 7), (ADD, 11, 10, 2, 0), (MULADD, 12, 0, 3, 8), (ADD, 13, 12, 2, 0)]
    graph = {"constants": None, "rotations": [0], "reads": reads, "ops": ops, "values_len": 14, "beta_idx": 2,
             "theta_idx": 3, "trash_challenge_idx": 4, "y_idx": 5, "previous_value_idx": 6, "result_idx": 13}
    return graph, (1, 11, 13, 9)


def multi_lookup_graphs():
    """A lookup of three input expressions in two helper chunks, the table the
    theta-compression of (f3, f4) at rotations 0 and +1, selector f5 * a2:
      chunk 0: f_0 = (a0, a1(+1)) compressed, f_1 = a2 f0      -> product, sum of partial products
      chunk 1: f_2 = a1 - a0(-1)
    Returns [(graph, outputs)] per chunk; every chunk computes table and selector."""
    def common(reads, ops, first_free):
        t = first_free
        reads = reads + [(FIXED, 3, 0, t), (FIXED, 4, 1, t + 1), (FIXED, 5, 0, t + 2), (ADVICE, 2, 0, t + 3)]
        ops = ops + [(MULADD, t + 4, 0, 3, t), (MULADD, t + 5, t + 4, 3, t + 1), (ADD, t + 6, t + 5, 2, 0),
                     (MUL, t + 7, t + 2, t + 3, 0)]
        return reads, ops, t + 6, t + 7, t + 8
    # chunk 0: inputs f_0 = theta-compression of (a0, a1(+1)) + beta, f_1 = a2 f0 + beta
    r0 = [(ADVICE, 0, 0, 7), (ADVICE, 1, 1, 8), (ADVICE, 2, 0, 9), (FIXED, 0, 0, 10)]
    o0 = [(MULADD, 11, 0, 3, 7), (MULADD, 12, 11, 3, 8), (ADD, 13, 12, 2, 0),      # f_0 + beta
          (MUL, 14, 9, 10, 0), (MULADD, 15, 0, 3, 14), (ADD, 16, 15, 2, 0),        # f_1 + beta
          (MUL, 17, 13, 16, 0),                                                    # product
          (ADD, 18, 16, 13, 0)]                                                    # sum of partial products
    r0, o0, tbl0, sel0, n0 = common(r0, o0, 19)
    g0 = {"constants": None, "rotations": [0, 1, -1], "reads": r0, "ops": o0, "values_len": n0, "beta_idx": 2,
          "theta_idx": 3, "trash_challenge_idx": 4, "y_idx": 5, "previous_value_idx": 6, "result_idx": 17}
    # chunk 1: f_2 = a1 - a0(-1), + beta; one input: sum of partial products = 1
    r1 = [(ADVICE, 1, 0, 7), (ADVICE, 0, 2, 8)]
    o1 = [(SUB, 9, 7, 8, 0), (MULADD, 10, 0, 3, 9), (ADD, 11, 10, 2, 0)]
    r1, o1, tbl1, sel1, n1 = common(r1, o1, 12)
    g1 = {"constants": None, "rotations": [0, 1, -1], "reads": r1, "ops": o1, "values_len": n1, "beta_idx": 2,
          "theta_idx": 3, "trash_challenge_idx": 4, "y_idx": 5, "previous_value_idx": 6, "result_idx": 11}
    return [(g0, (18, 17, tbl0, sel0)), (g1, (1, 11, tbl1, sel1))]


def trash_graph():
    """A trash argument's compression of (a0 - f1, a1 a2(+1)) with the trash
    challenge (Horner from zero, evaluation.rs:776-785)."""
    reads = [(ADVICE, 0, 0, 7), (FIXED, 1, 0, 8), (ADVICE, 1, 0, 9), (ADVICE, 2, 1, 10)]
    ops = [(SUB, 11, 7, 8, 0), (MUL, 12, 9, 10, 0), (MULADD, 13, 0, 4, 11), (MULADD, 14, 13, 4, 12)]
    return {"constants": None, "rotations": [0, 1], "reads": reads, "ops": ops, "values_len": 15, "beta_idx": 2,
            "theta_idx": 3, "trash_challenge_idx": 4, "y_idx": 5, "previous_value_idx": 6, "result_idx": 14}


def with_constants(graph, zero, one):
    """The graph with GraphEvaluator's first constants [0, 1] filled in."""
    g = dict(graph)
    g["constants"] = [zero, one]
    return g
