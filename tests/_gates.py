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
